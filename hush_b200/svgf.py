"""Host-side mirror of the reference's ``SVGF`` class (src/denoise/svgf.js:273-379, src/index.d.ts:63-83)."""
from __future__ import annotations

import ctypes as C
from typing import Optional

from . import _lib as L
from .hush import HushError, _FIELD, _stream_handle, device_view

SVGF_INPUTS = ["radiance", "normalDepth", "motion", "material", "emission", "prevNormalDepth", "prevMotion"]
_OPT_FIELDS = {"iterations": "iterations", "sigmaL": "sigma_l", "sigmaN": "sigma_n", "sigmaZ": "sigma_z",
               "alphaColor": "alpha_color", "alphaMoments": "alpha_moments", "taaAlpha": "taa_alpha", "taa": "taa"}


class SVGF:
    """``SVGF(device, width, height, options)``: SVGF + TAA, same G-buffer as Hush plus last frame's normalDepth and
    motion (svgf.js:341)."""

    def __init__(self, device=None, width: int = 0, height: int = 0, options: Optional[dict] = None):
        import torch

        o = L.lib().svgf_options_default()
        for k, v in (options or {}).items():
            if k not in _OPT_FIELDS:
                raise HushError(f"SVGF: unknown option '{k}'")
            setattr(o, _OPT_FIELDS[k], int(v) if k in ("iterations", "taa") else float(v))
        dev = torch.cuda.current_device() if device is None else int(getattr(device, "index", device) or 0)
        h = C.c_void_p()
        rc = L.lib().svgf_create(int(width), int(height), C.byref(o), dev, C.byref(h))
        if rc != L.HUSH_OK:
            raise HushError(L.lib().svgf_last_error(None).decode())
        self._h = h
        self._w, self._hgt = int(width), int(height)
        self._inp = L.SvgfInputs()

    @property
    def width(self) -> int:
        return self._w

    @property
    def height(self) -> int:
        return self._hgt

    def encode(self, inputs: dict, timer=None, stream=None):
        for k, name in enumerate(SVGF_INPUTS):
            t = inputs.get(name)
            if t is None:
                raise HushError(f"SVGF.encode: missing input '{name}'")
            if not t.is_cuda or t.dtype.itemsize != 2 or t.dim() != 3 or t.shape[2] != 4:
                raise HushError(f"SVGF.encode: '{name}' must be a CUDA (H, W, 4) float16 tensor")
            if t.shape[0] != self._hgt or t.shape[1] != self._w:
                raise HushError(f"SVGF.encode: '{name}' is {t.shape[1]}x{t.shape[0]}, the denoiser "
                                f"{self._w}x{self._hgt} (call resize)")
            setattr(self._inp, _FIELD[name], t.data_ptr())
            self._inp.pitch[k] = t.stride(0) * 2
        out = C.c_void_p()
        rc = L.lib().svgf_encode(self._h, C.byref(self._inp), C.c_void_p(_stream_handle(stream)), C.byref(out))
        if rc != L.HUSH_OK:
            raise HushError(L.lib().svgf_last_error(self._h).decode())
        return device_view(out.value, self._hgt, self._w)

    denoise = encode

    @property
    def output(self):
        return device_view(L.lib().svgf_output(self._h), self._hgt, self._w)

    def resize(self, width: int, height: int):
        rc = L.lib().svgf_resize(self._h, int(width), int(height))
        if rc != L.HUSH_OK:
            raise HushError(L.lib().svgf_last_error(self._h).decode())
        self._w, self._hgt = int(width), int(height)

    def reset(self):
        L.lib().svgf_reset(self._h)

    def destroy(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().svgf_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.destroy()
        except Exception:
            pass
