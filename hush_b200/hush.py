"""Host-side mirror of the reference's ``Hush`` class (src/denoise/hush.js:719-875, src/index.d.ts:36-61).

Device buffers replace GPUTextures: inputs are CUDA tensors of shape (H, W, 4) and dtype float16 (rgba16float);
the output is a zero-copy (H, W, 4) float16 view of an instance-owned buffer that alternates between two images
from frame to frame, like the reference's output texture (hush.js:796-798). A CUDA stream replaces the command
encoder: work is enqueued on ``stream`` (default: torch's current stream).

Every call goes through the C ABI of libhush_b200.so; there is no CPU or PyTorch fallback. Errors raise
``HushError`` with the reference's messages (hush.js:735, 743, 765, 816, 818).
"""
from __future__ import annotations

import base64
import ctypes as C
import os
from typing import Optional

import numpy as np

from . import _lib as L

INPUTS = ["radiance", "normalDepth", "motion", "material", "emission"]  # hush.js:723
N_FEAT, N_OUT = 20, 12  # hush.js:18-19
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "hush-weights.bin")


class HushError(RuntimeError):
    """An error raised by the denoiser (the reference throws ``Error`` with the same text)."""


def hiddenOf(n: int) -> int:  # noqa: N802 (reference name)
    """Hidden width h of the MLP for n f16 weights, n = h^2 + 34 h + 12 (hush.js:22-25); 0 if none fits."""
    return int(L.lib().hush_hidden_of(int(n)))


def decode_weights(w) -> np.ndarray:
    """decodeWeights (hush.js:713-717): base64 string, bytes-like, numpy / typed array -> uint16 f16 bit patterns."""
    if isinstance(w, str):
        w = base64.b64decode(w)
    if isinstance(w, (bytes, bytearray, memoryview)):
        return np.frombuffer(bytes(w), dtype="<u2").copy()
    try:
        import torch

        if isinstance(w, torch.Tensor):
            w = w.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    a = np.asarray(w)
    if a.dtype == np.float16:
        return a.view(np.uint16).reshape(-1).copy()
    if a.dtype == np.uint16:
        return a.reshape(-1).copy()
    return np.frombuffer(a.tobytes(), dtype="<u2").copy()


def builtin_weights() -> np.ndarray:
    """The reference's built-in weights (hush-weights.bin: 812 f16 values, h = 16)."""
    return np.fromfile(WEIGHTS_PATH, dtype="<u2")


def _check(rc: int, handle=None):
    if rc != L.HUSH_OK:
        msg = L.lib().hush_last_error(handle) if handle else L.lib().hush_global_error()
        raise HushError((msg or b"").decode() or f"hush error {rc}")


def _stream_handle(stream) -> Optional[int]:
    import torch

    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


class _DevView:
    """A (H, W, 4) float16 view of device memory for torch.as_tensor (``__cuda_array_interface__``)."""

    def __init__(self, ptr: int, h: int, w: int, c: int = 4, typestr: str = "<f2"):
        self.__cuda_array_interface__ = {"shape": (h, w, c), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def device_view(ptr: int, h: int, w: int, c: int = 4, typestr: str = "<f2"):
    import torch

    return torch.as_tensor(_DevView(ptr, h, w, c, typestr), device="cuda")


def _fill_inputs(inp: "L.HushInputs", tensors: dict, names=INPUTS):
    for k, name in enumerate(names):
        t = tensors.get(name) if tensors is not None else None
        if t is None:
            setattr(inp, _FIELD[name], None)
            continue
        if not t.is_cuda or t.dtype.itemsize != 2 or t.dim() != 3 or t.shape[2] != 4:
            raise HushError(f"Hush.denoise: '{name}' must be a CUDA (H, W, 4) float16 tensor (rgba16float)")
        if t.stride(2) != 1 or t.stride(1) != 4:
            raise HushError(f"Hush.denoise: '{name}' must have contiguous texels (strides (*, 4, 1))")
        setattr(inp, _FIELD[name], t.data_ptr())
        inp.width[k] = t.shape[1]
        inp.height[k] = t.shape[0]
        inp.pitch[k] = t.stride(0) * 2


MLP_MODES = {"fp32": L.MLP_FP32, "bf16": L.MLP_BF16, "f16": L.MLP_F16, "half": L.MLP_HALF}

_FIELD = {"radiance": "radiance", "normalDepth": "normal_depth", "motion": "motion", "material": "material",
          "emission": "emission", "prevNormalDepth": "prev_normal_depth", "prevMotion": "prev_motion"}


class Hush:
    """Drop-in ``Hush``: ``Hush(device, {"width", "height", "exposure", "weights", "f16"})``.

    ``f16=True`` is the reference's option: the MLP in f16 arithmetic (``mlp="half"``). Extra options of this
    implementation: ``mlp`` ("fp32" | "bf16" | "f16" | "half"; "bf16" / "f16" are the split-precision tensor-core
    forms, "half" the reference's f16 arithmetic, "fp32" the reference's default),
    ``schedule`` ("fused" | "passes"), ``graph`` (replay whole frames as CUDA graphs).
    """

    # hush.js:721 asks for 8 storage textures per stage; the CUDA equivalent is an sm_100a device
    requiredLimits = {"computeCapability": (10, 0), "maxSharedMemoryPerBlockOptin": 100 * 1024}

    def __init__(self, device=None, options: Optional[dict] = None, **kw):
        import torch

        opts = dict(options or {})
        opts.update(kw)
        width, height = opts.get("width"), opts.get("height")
        if device is None:
            dev = torch.cuda.current_device()
        elif isinstance(device, torch.device):
            dev = device.index if device.index is not None else torch.cuda.current_device()
        else:
            dev = int(device)
        self.device = dev
        d = L.lib().hush_desc_default(int(width or 0), int(height or 0))
        d.exposure = float(opts.get("exposure", 1.0))
        d.device = dev
        w = opts.get("weights")
        self._wbuf = None
        if w is not None:
            self._wbuf = np.ascontiguousarray(decode_weights(w))
            d.weights = self._wbuf.ctypes.data_as(C.POINTER(C.c_uint16))
            d.n_weights = self._wbuf.size
        d.f16 = 1 if opts.get("f16", False) else 0
        d.mlp_mode = MLP_MODES[opts.get("mlp", "fp32")]
        d.schedule = {"fused": L.SCHED_FUSED, "passes": L.SCHED_PASSES}[opts.get("schedule", "fused")]
        h = C.c_void_p()
        _check(L.lib().hush_create(C.byref(d), C.byref(h)))
        self._h = h
        if opts.get("graph"):
            _check(L.lib().hush_set_graph(self._h, 1), self._h)
        self._inp = L.HushInputs()

    # ---------------------------------------------------------------------------------------------- properties
    @property
    def width(self) -> int:
        w, h = C.c_int(), C.c_int()
        L.lib().hush_get_size(self._h, C.byref(w), C.byref(h))
        return w.value

    @property
    def height(self) -> int:
        w, h = C.c_int(), C.c_int()
        L.lib().hush_get_size(self._h, C.byref(w), C.byref(h))
        return h.value

    @property
    def hidden(self) -> int:
        return L.lib().hush_get_hidden(self._h)

    @property
    def frame(self) -> int:
        return L.lib().hush_get_frame(self._h)

    @property
    def exposure(self) -> float:
        return float(L.lib().hush_get_exposure(self._h))

    @exposure.setter
    def exposure(self, e: float):
        _check(L.lib().hush_set_exposure(self._h, float(e)), self._h)

    @property
    def handle(self) -> int:
        return self._h.value

    # ---------------------------------------------------------------------------------------------- methods
    def denoise(self, inputs: dict, timer=None, stream=None):
        """Enqueues one frame; returns the output image, a (H, W, 4) float16 view (hush.js:813-822)."""
        if inputs is None:
            raise HushError("Hush.denoise: missing inputs")
        for name in INPUTS:
            if inputs.get(name) is None:
                raise HushError(f"Hush.denoise: missing input '{name}'")
        _fill_inputs(self._inp, inputs)
        if timer is not None:
            _check(L.lib().hush_timer_enable(self._h, 2 if getattr(timer, "span", False) else 1), self._h)
        out = C.c_void_p()
        _check(L.lib().hush_denoise(self._h, C.byref(self._inp), C.c_void_p(_stream_handle(stream)), C.byref(out)),
               self._h)
        if timer is not None:
            timer.record(self.timings())
            L.lib().hush_timer_enable(self._h, 0)
        return device_view(out.value, self.height, self.width)

    def denoise_host(self, inputs: dict, out=None, stream=None):
        """One frame with the G-buffer in host memory: (H, W, 4) float16 CPU tensors (pinned for asynchronous
        copies) in, the output copied into `out` (a CPU float16 tensor, allocated pinned if None). Calls overlap
        their copies with the previous frame's kernels; `out` is complete after host_join(stream) and a synchronize
        (hush_denoise_host / hush_host_join)."""
        import torch

        inp = L.HushInputs()
        for k, name in enumerate(INPUTS):
            t = inputs.get(name) if inputs is not None else None
            if t is None:
                raise HushError(f"Hush.denoise: missing input '{name}'")
            if t.is_cuda or t.dtype.itemsize != 2 or t.dim() != 3 or t.shape[2] != 4 or t.stride(2) != 1 \
                    or t.stride(1) != 4:
                raise HushError(f"Hush.denoise_host: '{name}' must be a host (H, W, 4) float16 tensor with dense rows")
            setattr(inp, _FIELD[name], t.data_ptr())
            inp.width[k], inp.height[k] = t.shape[1], t.shape[0]
            inp.pitch[k] = t.stride(0) * 2
        if out is None:
            out = torch.empty((self.height, self.width, 4), dtype=torch.float16).pin_memory()
        if out.is_cuda or out.dtype != torch.float16 or tuple(out.shape) != (self.height, self.width, 4) \
                or out.stride(1) != 4 or out.stride(2) != 1:
            raise HushError("Hush.denoise_host: out must be a host (H, W, 4) float16 tensor with dense rows")
        _check(L.lib().hush_denoise_host(self._h, C.byref(inp), out.data_ptr(), out.stride(0) * 2,
                                         C.c_void_p(_stream_handle(stream))), self._h)
        return out

    def host_join(self, stream=None):
        """`stream` waits for every output copy denoise_host enqueued."""
        _check(L.lib().hush_host_join(self._h, C.c_void_p(_stream_handle(stream))), self._h)

    def timings(self) -> list:
        """[(label, ms)] of the last timed frame (synchronises on its events)."""
        arr = (L.HushTiming * 16)()
        n = L.lib().hush_timer_read(self._h, arr, 16)
        if n < 0:
            _check(L.HUSH_ERR_CUDA, self._h)
        return [(arr[i].label.decode(), float(arr[i].ms)) for i in range(n)]

    @property
    def output(self):
        """Output of the last denoise() (hush.js:798)."""
        p = L.lib().hush_output(self._h)
        return device_view(p, self.height, self.width)

    def resize(self, width: int, height: int):
        """Reallocates for a new size and resets the history (hush.js:764-794)."""
        _check(L.lib().hush_resize(self._h, int(width), int(height)), self._h)

    def reset(self):
        """Drops the temporal history (hush.js:801)."""
        _check(L.lib().hush_reset(self._h), self._h)

    def kernel_status(self) -> int:
        """The kernels' error word (a bounded wait that gave up sets a bit; synchronises, then clears it): raises
        HushError if any bit was set."""
        w = C.c_uint()
        _check(L.lib().hush_kernel_status(self._h, C.byref(w)), self._h)
        return w.value

    def set_weights(self, weights):
        self._wbuf = np.ascontiguousarray(decode_weights(weights))
        _check(L.lib().hush_set_weights(self._h, self._wbuf.ctypes.data_as(C.POINTER(C.c_uint16)),
                                         self._wbuf.size), self._h)

    def set_mlp(self, mode: str):
        _check(L.lib().hush_set_mlp_mode(self._h, MLP_MODES[mode]), self._h)

    def set_schedule(self, schedule: str):
        _check(L.lib().hush_set_schedule(self._h, {"fused": 0, "passes": 1}[schedule]), self._h)

    def set_graph(self, enable: bool):
        _check(L.lib().hush_set_graph(self._h, 1 if enable else 0), self._h)

    def destroy(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().hush_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.destroy()
        except Exception:
            pass

    # ---------------------------------------------------------------------------------------------- pass level
    def run_pass(self, name: str, inputs: Optional[dict] = None, stream=None):
        """Runs one reference pass on the instance state (tests and adjoint checks)."""
        p = L.PASS_NAMES.index(name)
        if inputs is not None:
            _fill_inputs(self._inp, inputs)
        _check(L.lib().hush_run_pass(self._h, p, C.byref(self._inp) if inputs is not None else None,
                                     C.c_void_p(_stream_handle(stream))), self._h)

    def end_frame(self):
        _check(L.lib().hush_end_frame(self._h), self._h)

    def buffer(self, name: str):
        """A state image as a (h, w, 4) float16 view, or (h, w, 8) for the packed feature images F0..F3."""
        ptr, w, h, tb = C.c_void_p(), C.c_int(), C.c_int(), C.c_int()
        _check(L.lib().hush_buffer(self._h, L.BUF[name], C.byref(ptr), C.byref(w), C.byref(h), C.byref(tb)), self._h)
        return device_view(ptr.value, h.value, w.value, tb.value // 2)


class HushTimer:
    """Per-pass (default) or whole-frame (``span=True``) GPU timer, like src/gpu.js GpuTimer."""

    def __init__(self, span: bool = False):
        self.span = span
        self.last = []

    def record(self, timings):
        self.last = timings
