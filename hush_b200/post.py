"""The demo's display post (src/demo/post.js) on a headless device buffer: split-screen composite of two or three
linear HDR images, six-level bloom, vignette, AgX tone mapping, sRGB and the divider line.

    post = Post(0, "rgba8unorm", bloom=0.03, vignette=0.35)     # new Post(device, format, {bloom, vignette})
    img = post.encode(left=hush_out, right=svgf_out, split=0.5)  # (H, W, 4) uint8 CUDA tensor

The reference renders into a canvas texture; here the target is a CUDA tensor (uint8 for "rgba8unorm" /
"bgra8unorm", float32 for "rgba32float"), allocated at the input size unless one is passed.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

from . import _lib as L
from .hush import HushError, _DevView, _stream_handle

FORMATS = {"rgba8unorm": L.POST_RGBA8, "bgra8unorm": L.POST_BGRA8, "rgba32float": L.POST_RGBA32F}


def _image(t, name, shape=None):
    if t is None:
        return None
    if not t.is_cuda or t.dtype.itemsize != 2 or t.dim() != 3 or t.shape[2] != 4 or not t.is_contiguous():
        raise HushError(f"Post.encode: '{name}' must be a contiguous CUDA (H, W, 4) float16 tensor")
    if shape is not None and tuple(t.shape[:2]) != shape:
        raise HushError(f"Post.encode: '{name}' is {t.shape[1]}x{t.shape[0]}, expected {shape[1]}x{shape[0]}")
    return t


class Post:
    """new Post(device, format, {bloom, vignette}) (post.js:137-156)."""

    def __init__(self, device=None, format: str = "rgba8unorm", options: Optional[dict] = None, **kw):
        import torch

        opts = dict(options or {})
        opts.update(kw)
        if format not in FORMATS:
            raise HushError(f"Post: unknown target format '{format}' (one of {', '.join(FORMATS)})")
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.format = format
        d = L.lib().hush_post_desc_default()
        d.device = self.device
        d.format = FORMATS[format]
        self._bloom = float(opts.get("bloom", d.bloom))
        self._vignette = float(opts.get("vignette", d.vignette))
        d.bloom, d.vignette = self._bloom, self._vignette
        h = C.c_void_p()
        if L.lib().hush_post_create(C.byref(d), C.byref(h)) != L.HUSH_OK:
            raise HushError(L.lib().hush_post_last_error(None).decode())
        self._h = h

    @property
    def bloom(self) -> float:
        return self._bloom

    @bloom.setter
    def bloom(self, v: float):
        self._bloom = float(v)
        L.lib().hush_post_set(self._h, self._bloom, self._vignette)

    @property
    def vignette(self) -> float:
        return self._vignette

    @vignette.setter
    def vignette(self, v: float):
        self._vignette = float(v)
        L.lib().hush_post_set(self._h, self._bloom, self._vignette)

    def encode(self, left, right, mid=None, split: float = 0.5, split2: Optional[float] = None, same: bool = False,
               exposure: float = 1.0, target=None, width: Optional[int] = None, height: Optional[int] = None,
               line: float = 1.5, stream=None):
        """Post.encode (post.js:191-210). Returns the target tensor (height, width, 4)."""
        import torch

        left = _image(left, "left")
        hw = tuple(left.shape[:2])
        right = _image(right, "right", hw)
        mid = _image(mid, "mid", hw)
        width = int(width or (target.shape[1] if target is not None else hw[1]))
        height = int(height or (target.shape[0] if target is not None else hw[0]))
        dt = torch.float32 if self.format == "rgba32float" else torch.uint8
        if target is None:
            target = torch.empty((height, width, 4), dtype=dt, device=f"cuda:{self.device}")
        elif (not target.is_cuda or target.dtype != dt or tuple(target.shape) != (height, width, 4)
              or target.stride(1) != 4 or target.stride(2) != 1):
            raise HushError(f"Post.encode: target must be a CUDA ({height}, {width}, 4) {dt} tensor with dense rows")
        inp = L.HushPostInputs(left.data_ptr(), right.data_ptr(), mid.data_ptr() if mid is not None else None,
                               hw[1], hw[0], float(split), float(split if split2 is None else split2),
                               float(exposure), float(line), 1 if same else 0)
        pitch = target.stride(0) * target.element_size()
        rc = L.lib().hush_post_encode(self._h, C.byref(inp), target.data_ptr(), width, height, pitch,
                                      C.c_void_p(_stream_handle(stream)))
        if rc != L.HUSH_OK:
            raise HushError(L.lib().hush_post_last_error(self._h).decode())
        return target

    def buffer(self, level: int):
        """Level 0: the composited HDR image; 1..6: the bloom levels of the last encode (float16 views)."""
        import torch

        w, h = C.c_int(), C.c_int()
        p = L.lib().hush_post_buffer(self._h, int(level), C.byref(w), C.byref(h))
        if not p:
            raise HushError(f"Post.buffer: no level {level} (encode first; levels 0..{L.POST_LEVELS})")
        return torch.as_tensor(_DevView(p, h.value, w.value, 4, "<f2"), device=f"cuda:{self.device}")

    def destroy(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().hush_post_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.destroy()
        except Exception:
            pass
