"""Learned FSAI preconditioner: model handle, weight files and training.

The network, its Kaporin objective and its forward/backward kernels live in
libtptfem.so (csrc/lfsai.cu); this module drives them: loss/gradient/Adam steps
on the device and a versioned weight file.

Weight file (little endian): 8-byte magic b"TPTLFSAI", u32 version (2), u32
parameter count, then that many float32 values.
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np

from . import _native as N

MAGIC = b"TPTLFSAI"
VERSION = 2


def param_count():
    return int(N.load().tptfem_lfsai_param_count())


class LearnedFsai:
    """A device-resident network (tptfem_lfsai) on `ctx`'s GPU."""

    def __init__(self, ctx, seed=0, params=None):
        self.ctx = ctx
        self.lib = ctx.lib
        h = C.c_void_p()
        ctx.check(self.lib.tptfem_lfsai_create(ctx.h, int(seed), C.byref(h)))
        self.h = h
        self.n_params = param_count()
        if params is not None:
            self.set_params(params)

    def get_params(self):
        p = np.zeros(self.n_params, np.float32)
        self.ctx.check(self.lib.tptfem_lfsai_get_params(self.ctx.h, self.h, N.ptr(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.size}")
        self.ctx.check(self.lib.tptfem_lfsai_set_params(self.ctx.h, self.h, N.ptr(p)))

    def loss(self, system, grad=False):
        """Kaporin loss (1/n) sum_i log q_i on `system` (and, with grad=True, the accumulated gradient)."""
        out = C.c_double()
        g = np.zeros(self.n_params, np.float32) if grad else None
        self.ctx.check(self.lib.tptfem_lfsai_loss(self.ctx.h, self.h, system.h, int(grad), C.byref(out),
                                                  N.ptr(g) if grad else None))
        return (out.value, g) if grad else out.value

    def adam(self, lr, clip=1.0):
        self.ctx.check(self.lib.tptfem_lfsai_adam(self.ctx.h, self.h, float(lr), float(clip)))

    def attach(self, system):
        self.ctx.check(self.lib.tptfem_system_attach_lfsai(self.ctx.h, system.h, self.h))

    def save(self, path):
        p = self.get_params()
        with open(path, "wb") as f:
            f.write(MAGIC + struct.pack("<II", VERSION, p.size) + p.astype("<f4").tobytes())

    @classmethod
    def load(cls, ctx, path):
        return cls(ctx, params=read_weights(path))

    def __del__(self):
        if getattr(self, "h", None) is not None and self.ctx.h:
            self.lib.tptfem_lfsai_free(self.h)
            self.h = None


def read_weights(path):
    data = open(path, "rb").read()
    if data[:8] != MAGIC:
        raise ValueError(f"{path}: not a learned-FSAI weight file")
    version, count = struct.unpack("<II", data[8:16])
    if version != VERSION:
        raise ValueError(f"{path}: weight file version {version}, expected {VERSION}")
    p = np.frombuffer(data[16:16 + 4 * count], dtype="<f4").astype(np.float32)
    if count != param_count():
        raise ValueError(f"{path}: {count} parameters, the library's network has {param_count()}")
    return p
