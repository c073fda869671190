"""Neural radiance cache (include/illume_gpu.h, ilm_nrc_*).

Inputs are (n, 12) float32 rows: position, outgoing direction, normal,
albedo.  Outputs are (n, 3) RGB radiance.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import CUDA_STREAM_LEGACY, ptr
from .primitive import Context

N_PARAMS = 30720
LAYERS = [(64, 208), (64, 64), (64, 64), (64, 64), (64, 64), (16, 64)]   # (out, in)


class ilm_nrc_config(ctypes.Structure):
    _fields_ = [("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float),
                ("eps", ctypes.c_float), ("seed", ctypes.c_uint64), ("bound", ctypes.c_float * 6),
                ("ema", ctypes.c_float), ("weight_decay", ctypes.c_float)]


def split_params(p: np.ndarray):
    """Flat master weights -> list of (out, in) matrices."""
    out, off = [], 0
    for o, i in LAYERS:
        out.append(p[off: off + o * i].reshape(o, i))
        off += o * i
    return out


class RadianceCache:
    def __init__(self, ctx: Context, bound, lr=1e-2, beta1=0.9, beta2=0.99, eps=1e-10, seed=4, ema=0.99,
                 weight_decay=1.0):
        """`ema`: inference uses a moving average of the weights over Adam
        steps with this decay (0 = the latest weights).  `weight_decay`:
        decoupled weight decay (AdamW), each step also subtracting
        lr * weight_decay * w (0 = plain Adam); it keeps the online-trained
        cache smooth."""
        self.ctx = ctx
        if hasattr(bound, "min") and hasattr(bound, "max"):      # Bounds3f
            bound = tuple(bound.min) + tuple(bound.max)
        c = ilm_nrc_config(lr, beta1, beta2, eps, seed)
        for k in range(6):
            c.bound[k] = bound[k]
        c.ema = ema
        c.weight_decay = weight_decay
        h = ctypes.c_void_p()
        ctx.check(ctx._lib.ilm_nrc_create(ctx.handle, ctypes.addressof(c), ctypes.byref(h)), "ilm_nrc_create")
        self.handle = h

    def params(self) -> np.ndarray:
        p = np.empty(N_PARAMS, np.float32)
        self.ctx.check(self.ctx._lib.ilm_nrc_params(self.ctx.handle, self.handle, ptr(p), None), "ilm_nrc_params")
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        self.ctx.check(self.ctx._lib.ilm_nrc_params(self.ctx.handle, self.handle, None, ptr(p)), "ilm_nrc_params")

    def infer(self, inputs, out=None, stream=None):
        n = _rows(inputs)
        if out is None:
            out = np.empty((n, 3), np.float32)
        self.ctx.check(self.ctx._lib.ilm_nrc_infer(self.ctx.handle, self.handle, ptr(inputs), n, ptr(out),
                                                   _stream(stream, inputs)), "ilm_nrc_infer")
        return out

    def train_step(self, inputs, targets, stream=None, with_loss: bool = True):
        """One Adam step; returns the batch loss, or None without waiting for
        the step when with_loss is False."""
        loss = ctypes.c_float()
        self.ctx.check(self.ctx._lib.ilm_nrc_train_step(self.ctx.handle, self.handle, ptr(inputs), ptr(targets),
                                                        _rows(inputs), ctypes.byref(loss) if with_loss else None,
                                                        _stream(stream, inputs)),
                       "ilm_nrc_train_step")
        return loss.value if with_loss else None

    def gradients(self, inputs, targets):
        g = np.empty(N_PARAMS, np.float32)
        loss = ctypes.c_float()
        self.ctx.check(self.ctx._lib.ilm_nrc_gradients(self.ctx.handle, self.handle, ptr(inputs), ptr(targets),
                                                       _rows(inputs), ptr(g), ctypes.byref(loss)),
                       "ilm_nrc_gradients")
        return g, loss.value

    def encode(self, inputs) -> np.ndarray:
        """bf16 encodings as float32 (n, 208)."""
        n = _rows(inputs)
        raw = np.empty((n, 208), np.uint16)
        self.ctx.check(self.ctx._lib.ilm_nrc_encode(self.ctx.handle, self.handle, ptr(inputs), n, ptr(raw)),
                       "ilm_nrc_encode")
        return (raw.astype(np.uint32) << 16).view(np.float32)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.ctx._lib.ilm_nrc_destroy(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _rows(a) -> int:
    if isinstance(a, np.ndarray):
        return a.size // 12 if a.shape[-1] == 12 else a.shape[0]
    return a.shape[0]


def _stream(stream, buf=None):
    """As primitive._stream: torch's current stream for torch CUDA tensors
    when no stream is given, NULL (the context's stream) for host arrays."""
    if stream is None:
        if getattr(buf, "is_cuda", False):
            import torch
            h = torch.cuda.current_stream(buf.device).cuda_stream
            # torch's default stream is the legacy default stream, handle 0;
            # the C ABI reads NULL as the context's stream, so name it by
            # its explicit handle, cudaStreamLegacy (0x1)
            return h if h else CUDA_STREAM_LEGACY
        return None
    return stream if isinstance(stream, int) else stream.cuda_stream
