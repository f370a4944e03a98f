"""Device-buffer helpers for the GPU parity tests (all through the C ABI)."""
from __future__ import annotations

import ctypes

import numpy as np

import benchntt_b200 as bn


class DevBuf:
    """Device buffer owned by a bntt context (bntt_dev_alloc / bntt_dev_free)."""

    def __init__(self, ctx: bn.Context, nbytes: int):
        self.ctx = ctx
        self.nbytes = nbytes
        self.ptr = ctypes.c_void_p()
        bn.check(bn.lib().bntt_dev_alloc(ctx.handle, ctypes.byref(self.ptr), nbytes))

    @classmethod
    def from_array(cls, ctx: bn.Context, a: np.ndarray) -> "DevBuf":
        a = np.ascontiguousarray(a, dtype=np.uint64)
        d = cls(ctx, a.nbytes)
        bn.check(bn.lib().bntt_copy_h2d(ctx.handle, d.ptr, a.ctypes.data, a.nbytes))
        return d

    def to_array(self, rows: int | None = None) -> np.ndarray:
        rows = self.nbytes // 16 if rows is None else rows
        out = np.empty((rows, 2), dtype=np.uint64)
        self.ctx.synchronize()
        bn.check(bn.lib().bntt_copy_d2h(self.ctx.handle, out.ctypes.data, self.ptr, rows * 16))
        return out

    @property
    def addr(self) -> int:
        return self.ptr.value

    def free(self) -> None:
        if self.ptr:
            bn.check(bn.lib().bntt_dev_free(self.ctx.handle, self.ptr))
            self.ptr = ctypes.c_void_p()


def dev_blas(ctx, op, a: np.ndarray, b: np.ndarray, q: int, mu: int, x: int = 0,
             layout: int = bn.LAYOUT_HILO) -> np.ndarray:
    da, db = DevBuf.from_array(ctx, a), DevBuf.from_array(ctx, b)
    dc = DevBuf(ctx, a.nbytes)
    m = bn.modulus(q, mu)
    fn = getattr(bn.lib(), f"bntt_{op}_dev")
    n = a.size // 2
    if op == "axpy":
        bn.check(fn(ctx.handle, dc.ptr, da.ptr, db.ptr, bn.U128.of(x), n, ctypes.byref(m), layout))
    else:
        bn.check(fn(ctx.handle, dc.ptr, da.ptr, db.ptr, n, ctypes.byref(m), layout))
    out = dc.to_array(n)
    for d in (da, db, dc):
        d.free()
    return out


def hilo_to_u128(a: np.ndarray) -> np.ndarray:
    """hi-first pairs -> native little-endian __int128 layout (lo first)."""
    return np.ascontiguousarray(a[:, ::-1])


def u128_to_hilo(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a[:, ::-1])
