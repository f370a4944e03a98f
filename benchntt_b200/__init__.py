"""benchntt_b200 -- Python binding of libbntt (B200 / sm_100a).

libbntt implements benchNTT's 128-bit modular NTT and BLAS-style vector ops
with results identical to the reference scalar path (src/ntt_scalar.c,
src/blas_scalar.c).  This module is a thin ctypes layer over the C ABI in
include/bntt.h; every computation runs in the CUDA library.  There is no CPU
fallback: if libbntt.so is missing or cannot be loaded, importing the
functions that compute raises.

Array convention: residues are (n, 2) uint64 numpy arrays of hi-first pairs
(row i = high word, low word), the layout of the reference's data files
(src/config.c:29-30), or CUDA tensors of the same bytes (torch.uint64 or
int64, shape (n, 2)) for the device entry points.

Reference-shaped functions (argument order as in the reference):
    ntt(Y, X, modulus, mu, twiddles)        src/ntt_scalar.c:582
    vector_add(c, a, b, m)                  src/blas_scalar.c:578
    vector_sub(c, a, b, m)                  src/blas_scalar.c:586
    vector_mul(c, a, b, m, mu)              src/blas_scalar.c:594
    axpy(c, a, b, x, m, mu)                 src/blas_scalar.c:602
where modulus / mu / m / x are Python ints.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbntt.so")

OK, EINVAL, ENOMEM, EBUDGET, ECUDA, ETIMEOUT, ENODEV, EBUSY = range(8)
LAYOUT_HILO, LAYOUT_U128 = 0, 1
ARITH_AUTO, ARITH_REFERENCE = 0, 1

# Moduli of the reference programs.
Q_NTT = (1152921504606846975 << 64) | 18446744073709550897   # src/ntt_scalar.c:633
MU_NTT = (9223372036854775808 << 64) | 5752                  # src/ntt_scalar.c:632
Q_BLAS = (0x0FFFFFFFFFFFFFFF << 64) | 0xFFFFFFFFFFFFFFC5     # src/blas_scalar.c:27
MU_BLAS = (0x8000000000000000 << 64) | 0x1D8                 # src/blas_scalar.c:30


class BnttError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"bntt status {status}: {message}")
        self.status = status


class U128(ctypes.Structure):
    _fields_ = [("hi", ctypes.c_uint64), ("lo", ctypes.c_uint64)]

    @classmethod
    def of(cls, v: int) -> "U128":
        return cls((v >> 64) & 0xFFFFFFFFFFFFFFFF, v & 0xFFFFFFFFFFFFFFFF)


class ModulusC(ctypes.Structure):
    _fields_ = [("q", U128), ("mu", U128)]


class JobC(ctypes.Structure):
    _fields_ = [("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("plan", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class ServerConfigC(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("slots", ctypes.c_uint32),
                ("max_batch", ctypes.c_uint32)]


class RequestC(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("plan", ctypes.c_uint32), ("len", ctypes.c_uint64),
                ("x", ctypes.c_void_p), ("b", ctypes.c_void_p), ("scalar", U128),
                ("tag", ctypes.c_uint64), ("t_arrive", ctypes.c_double)]


class CompletionC(ctypes.Structure):
    _fields_ = [("tag", ctypes.c_uint64), ("y", ctypes.c_void_p), ("bytes", ctypes.c_size_t),
                ("t_arrive", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_done", ctypes.c_double), ("status", ctypes.c_int)]


class ServerStatsC(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("admission_waits", ctypes.c_uint64),
                ("peak_bytes", ctypes.c_size_t)]


REQ_NTT, REQ_VVMUL, REQ_AXPY = 0, 1, 2

_LIB = None

# (name, restype, argtypes)
_P, _S, _U64, _I, _U = (ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int,
                        ctypes.c_uint)
_PM = ctypes.POINTER(ModulusC)
_SIGS = [
    ("bntt_version", ctypes.c_char_p, []),
    ("bntt_last_error", ctypes.c_char_p, []),
    ("bntt_status_string", ctypes.c_char_p, [_I]),
    ("bntt_modulus_is_fast", _I, [_PM]),
    ("bntt_modulus_ntt_reference", ModulusC, []),
    ("bntt_modulus_blas_reference", ModulusC, []),
    ("bntt_ctx_create", _I, [ctypes.POINTER(_P), _I, _P]),
    ("bntt_ctx_destroy", _I, [_P]),
    ("bntt_ctx_synchronize", _I, [_P]),
    ("bntt_ctx_stream", _P, [_P]),
    ("bntt_ctx_set_arith", _I, [_P, _I]),
    ("bntt_ctx_set_hbm_budget", _I, [_P, _S]),
    ("bntt_ctx_hbm_in_use", _S, [_P]),
    ("bntt_ctx_sm_count", _I, [_P]),
    ("bntt_ctx_launch_count", _U64, [_P]),
    ("bntt_dev_alloc", _I, [_P, ctypes.POINTER(_P), _S]),
    ("bntt_dev_free", _I, [_P, _P]),
    ("bntt_copy_h2d", _I, [_P, _P, _P, _S]),
    ("bntt_copy_d2h", _I, [_P, _P, _P, _S]),
    ("bntt_fill_uniform_host", _I, [_P, _S, _U64, _U64, _PM, _I]),
    ("bntt_fill_uniform_dev", _I, [_P, _P, _S, _U64, _U64, _PM, _I]),
    ("bntt_plan_create", _I, [_P, ctypes.POINTER(_P), _U, _PM, _P, _I]),
    ("bntt_plan_create_dev", _I, [_P, ctypes.POINTER(_P), _U, _PM, _P, _I]),
    ("bntt_plan_destroy", _I, [_P]),
    ("bntt_ntt_prime", _I, [_U, _PM]),
    ("bntt_root_of_unity", _I, [_PM, _U, ctypes.POINTER(U128)]),
    ("bntt_powmod", _I, [_PM, U128, U128, ctypes.POINTER(U128)]),
    ("bntt_twiddles_negacyclic", _I, [_PM, _U, U128, _P, _I]),
    ("bntt_plan_create_negacyclic", _I, [_P, ctypes.POINTER(_P), _U, _PM, U128, _I]),
    ("bntt_plan_log2n", _U, [_P]),
    ("bntt_ntt_forward_dev", _I, [_P, _P, _P, _S]),
    ("bntt_ntt_forward_host", _I, [_P, _P, _P, _S]),
    ("bntt_ntt_forward_mul_dev", _I, [_P, _P, _P, _P, _I, _S]),
    ("bntt_ntt_inverse_dev", _I, [_P, _P, _P, _S]),
    ("bntt_batch_create", _I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), _S]),
    ("bntt_batch_destroy", _I, [_P]),
    ("bntt_batch_run_dev", _I, [_P, ctypes.POINTER(JobC), _S]),
    ("bntt_batch_run_host", _I, [_P, ctypes.POINTER(JobC), _S]),
    ("bntt_batch_run_host_async", _I, [_P, ctypes.POINTER(JobC), _S]),
    ("bntt_batch_sync", _I, [_P]),
    ("bntt_batch_run_percall_dev", _I, [_P, ctypes.POINTER(JobC), _S]),
    ("bntt_batch_run_dev_noalloc", _I, [_P, ctypes.POINTER(JobC), _S]),
    ("bntt_batch_status", _I, [_P]),
    ("bntt_batch_inject_wait_timeout", _I, [_P, ctypes.c_uint32]),
    ("bntt_batch_last_launches", _S, [_P]),
    ("bntt_batch_run_inverse_dev", _I, [_P, ctypes.POINTER(JobC), _S]),
    ("bntt_probe_imad_peak", _I, [_P, ctypes.POINTER(ctypes.c_double)]),
    ("bntt_probe_butterfly_peak", _I, [_P, ctypes.POINTER(ctypes.c_double)]),
    ("bntt_server_create", _I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), _S, _PM,
                                ctypes.POINTER(ServerConfigC)]),
    ("bntt_server_destroy", _I, [_P]),
    ("bntt_server_clock", ctypes.c_double, [_P]),
    ("bntt_server_submit", _I, [_P, ctypes.POINTER(RequestC)]),
    ("bntt_server_poll", _I, [_P, ctypes.POINTER(CompletionC), _S, ctypes.POINTER(_S)]),
    ("bntt_server_release", _I, [_P, _P]),
    ("bntt_server_drain", _I, [_P]),
    ("bntt_server_get_stats", _I, [_P, ctypes.POINTER(ServerStatsC)]),
    ("bntt_server_replay", _I, [_P, ctypes.POINTER(RequestC), _S, _I,
                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    ("bntt_server_replay_ex", _I, [_P, ctypes.POINTER(RequestC), _S, _I, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    ("bntt_split_by_cost", _I, [_P, _S, ctypes.c_uint32, _P]),
    ("bntt_multi_create", _I, [ctypes.POINTER(_P), ctypes.POINTER(_P), _S]),
    ("bntt_multi_destroy", _I, [_P]),
    ("bntt_multi_split", _I, [_P, ctypes.POINTER(JobC), _S, _P]),
    ("bntt_multi_run_host", _I, [_P, ctypes.POINTER(JobC), _S]),
    ("bntt_autotune", _I, [_P, ctypes.c_char_p]),
    ("bntt_autotune_load", _I, [_P, ctypes.c_char_p]),
    ("bntt_autotune_reset", _I, []),
] + [(f"bntt_{op}_{kind}", _I, [_P, _P, _P, _P, _S, _PM, _I])
     for op in ("vvadd", "vvsub", "vvmul") for kind in ("dev", "host")] + [
    (f"bntt_axpy_{kind}", _I, [_P, _P, _P, _P, U128, _S, _PM, _I]) for kind in ("dev", "host")]


def lib() -> ctypes.CDLL:
    """Loads libbntt.so (raises if it is missing: no fallback exists)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `make -C {_HERE}` "
                              "(or __graft_entry__.build())")
        l = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            fn = getattr(l, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _LIB = l
    return _LIB


def exported_symbols() -> list[str]:
    return [name for name, _, _ in _SIGS]


def check(status: int) -> None:
    if status != OK:
        raise BnttError(status, lib().bntt_last_error().decode(errors="replace"))


def modulus(q: int, mu: int | None = None) -> ModulusC:
    """Modulus struct; mu defaults to floor(2^251 / q) (MBITS = 124)."""
    if mu is None:
        mu = (1 << 251) // q
    return ModulusC(U128.of(q), U128.of(mu))


# ------------------------------------------------- NTT-friendly prime mode
def ntt_prime(log2_order: int) -> tuple[int, int]:
    """(q, mu): q = 2^124 - (c*2^log2_order - 1), smallest c giving a prime
    (Miller-Rabin, bntt_ntt_prime), mu = floor(2^251 / q)."""
    m = ModulusC()
    check(lib().bntt_ntt_prime(log2_order, ctypes.byref(m)))
    return (m.q.hi << 64) | m.q.lo, (m.mu.hi << 64) | m.mu.lo


def root_of_unity(q: int, mu: int, log2_order: int) -> int:
    """A primitive 2^log2_order-th root of unity mod q."""
    r = U128()
    check(lib().bntt_root_of_unity(ctypes.byref(modulus(q, mu)), log2_order, ctypes.byref(r)))
    return (r.hi << 64) | r.lo


def powmod(q: int, mu: int, a: int, e: int) -> int:
    r = U128()
    check(lib().bntt_powmod(ctypes.byref(modulus(q, mu)), U128.of(a), U128.of(e),
                            ctypes.byref(r)))
    return (r.hi << 64) | r.lo


def twiddles_negacyclic(q: int, mu: int, log2n: int, psi: int,
                        layout: int = LAYOUT_HILO) -> np.ndarray:
    """Host table T[k] = psi^brv(k) (T[0] = 1) as an (N, 2) uint64 array."""
    t = np.empty((1 << log2n, 2), dtype=np.uint64)
    check(lib().bntt_twiddles_negacyclic(ctypes.byref(modulus(q, mu)), log2n, U128.of(psi),
                                         t.ctypes.data, layout))
    return t


# ------------------------------------------------------------------ helpers
def pairs(a) -> np.ndarray:
    """View/convert to a C-contiguous (n, 2) uint64 array."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a.reshape(-1, 2)


def _host_ptr(a: np.ndarray) -> int:
    if not a.flags.c_contiguous:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data


def _is_cuda_tensor(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


def _dev_ptr(t) -> int:
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return t.data_ptr()


class Context:
    """A device, a stream and an HBM budget (bntt_ctx)."""

    def __init__(self, device: int = 0, stream: int | None = None, arith: int = ARITH_AUTO):
        self._h = ctypes.c_void_p()
        check(lib().bntt_ctx_create(ctypes.byref(self._h), device, stream))
        if arith != ARITH_AUTO:
            check(lib().bntt_ctx_set_arith(self._h, arith))
        self.device = device

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return lib().bntt_ctx_stream(self._h)

    def synchronize(self) -> None:
        check(lib().bntt_ctx_synchronize(self._h))

    def set_arith(self, arith: int) -> None:
        check(lib().bntt_ctx_set_arith(self._h, arith))

    def set_hbm_budget(self, nbytes: int) -> None:
        check(lib().bntt_ctx_set_hbm_budget(self._h, nbytes))

    @property
    def hbm_in_use(self) -> int:
        return lib().bntt_ctx_hbm_in_use(self._h)

    @property
    def sm_count(self) -> int:
        return lib().bntt_ctx_sm_count(self._h)

    @property
    def launches(self) -> int:
        return lib().bntt_ctx_launch_count(self._h)

    def autotune(self, path: str | None = None) -> None:
        """Times the compiled kernel shapes on this device and makes the
        fastest the defaults for plans / batches created afterwards."""
        check(lib().bntt_autotune(self._h, path.encode() if path else None))

    def autotune_load(self, path: str) -> None:
        check(lib().bntt_autotune_load(self._h, path.encode()))

    def imad_peak(self) -> float:
        """Measured 32-bit IMAD operations per second of this device."""
        v = ctypes.c_double()
        check(lib().bntt_probe_imad_peak(self._h, ctypes.byref(v)))
        return v.value

    def butterfly_peak(self) -> float:
        """Measured butterflies per second of the kernels' own butterfly on
        register-resident data (bntt_probe_butterfly_peak)."""
        v = ctypes.c_double()
        check(lib().bntt_probe_butterfly_peak(self._h, ctypes.byref(v)))
        return v.value

    def close(self) -> None:
        if self._h:
            lib().bntt_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """One transform size + modulus + device-resident twiddle table."""

    def __init__(self, ctx: Context, log2n: int, q: int, mu: int, twiddles,
                 layout: int = LAYOUT_HILO):
        self.ctx, self.log2n, self.q, self.mu, self.layout = ctx, log2n, q, mu, layout
        self._m = modulus(q, mu)
        self._h = ctypes.c_void_p()
        if _is_cuda_tensor(twiddles):
            self._tw_ref = twiddles
            check(lib().bntt_plan_create_dev(ctx.handle, ctypes.byref(self._h), log2n,
                                             ctypes.byref(self._m), _dev_ptr(twiddles), layout))
        else:
            tw = pairs(twiddles)
            if tw.shape[0] != 1 << log2n:
                raise ValueError(f"twiddle table must have {1 << log2n} entries")
            check(lib().bntt_plan_create(ctx.handle, ctypes.byref(self._h), log2n,
                                         ctypes.byref(self._m), _host_ptr(tw), layout))

    @classmethod
    def negacyclic(cls, ctx: Context, log2n: int, q: int, mu: int, psi: int,
                   layout: int = LAYOUT_HILO) -> "Plan":
        """Plan whose table T[k] = psi^brv(k) is generated on the device
        (bntt_plan_create_negacyclic): the network then computes the
        negacyclic NTT, outputs in bit-reversed order."""
        self = cls.__new__(cls)
        self.ctx, self.log2n, self.q, self.mu, self.layout = ctx, log2n, q, mu, layout
        self._m = modulus(q, mu)
        self._h = ctypes.c_void_p()
        check(lib().bntt_plan_create_negacyclic(ctx.handle, ctypes.byref(self._h), log2n,
                                                ctypes.byref(self._m), U128.of(psi), layout))
        return self

    @property
    def handle(self):
        return self._h

    def forward(self, y, x, batch: int | None = None) -> None:
        n = 1 << self.log2n
        if _is_cuda_tensor(x):
            b = batch if batch is not None else x.numel() // (2 * n)
            check(lib().bntt_ntt_forward_dev(self._h, _dev_ptr(y), _dev_ptr(x), b))
        else:
            b = batch if batch is not None else x.size // (2 * n)
            check(lib().bntt_ntt_forward_host(self._h, _host_ptr(y), _host_ptr(x), b))

    def inverse(self, x, y, batch: int | None = None) -> None:
        """x = ntt^-1(y) (bntt_ntt_inverse_dev); device tensors only."""
        n = 1 << self.log2n
        bt = batch if batch is not None else y.numel() // (2 * n)
        check(lib().bntt_ntt_inverse_dev(self._h, _dev_ptr(x), _dev_ptr(y), bt))

    def forward_mul(self, y, x, b, per_transform: bool = True, batch: int | None = None) -> None:
        """y = ntt(x) o b in one launch sequence (bntt_ntt_forward_mul_dev);
        device tensors only."""
        n = 1 << self.log2n
        bt = batch if batch is not None else x.numel() // (2 * n)
        check(lib().bntt_ntt_forward_mul_dev(self._h, _dev_ptr(y), _dev_ptr(x), _dev_ptr(b),
                                             1 if per_transform else 0, bt))

    def close(self) -> None:
        if self._h:
            lib().bntt_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Mixed-size transforms in one persistent work-queue kernel."""

    def __init__(self, ctx: Context, plans: list[Plan]):
        self.ctx, self.plans = ctx, plans
        arr = (ctypes.c_void_p * len(plans))(*[p.handle.value for p in plans])
        self._h = ctypes.c_void_p()
        check(lib().bntt_batch_create(ctx.handle, ctypes.byref(self._h), arr, len(plans)))

    @property
    def handle(self):
        return self._h

    @staticmethod
    def jobs(xs: list[int], ys: list[int], plan_ids: list[int]):
        arr = (JobC * len(xs))()
        for i, (x, y, p) in enumerate(zip(xs, ys, plan_ids)):
            arr[i].x, arr[i].y, arr[i].plan = x, y, p
        return arr

    def run_dev(self, jobs) -> None:
        check(lib().bntt_batch_run_dev(self._h, jobs, len(jobs)))

    def run_host(self, jobs) -> None:
        check(lib().bntt_batch_run_host(self._h, jobs, len(jobs)))

    def run_host_async(self, jobs) -> None:
        """Queue a host-buffer run; buffers stay untouched until sync()."""
        check(lib().bntt_batch_run_host_async(self._h, jobs, len(jobs)))

    def sync(self) -> None:
        check(lib().bntt_batch_sync(self._h))

    def run_inverse_dev(self, jobs) -> None:
        """Inverse transforms of the jobs (job.x -> job.y) in one launch."""
        check(lib().bntt_batch_run_inverse_dev(self._h, jobs, len(jobs)))

    def run_percall_dev(self, jobs) -> None:
        """Each job as its own launch(es): the per-call comparison path."""
        check(lib().bntt_batch_run_percall_dev(self._h, jobs, len(jobs)))

    def status(self) -> int:
        return lib().bntt_batch_status(self._h)

    @property
    def last_launches(self) -> int:
        return lib().bntt_batch_last_launches(self._h)

    def close(self) -> None:
        if self._h:
            lib().bntt_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def split_by_cost(logns, parts: int) -> np.ndarray:
    """bntt_split_by_cost: the owner (in [0, parts)) of each job of size
    2^logns[i], longest first to the least-loaded part.  Needs no GPU."""
    logns = np.ascontiguousarray(logns, dtype=np.uint32)
    owner = np.empty(len(logns), dtype=np.uint32)
    check(lib().bntt_split_by_cost(logns.ctypes.data, len(logns), parts, owner.ctypes.data))
    return owner


class Multi:
    """One job list over several batches (one per device, own plans each):
    split by cost, run from host buffers, no data exchanged between GPUs."""

    def __init__(self, batches: list[Batch]):
        self.batches = batches
        arr = (ctypes.c_void_p * len(batches))(*[b.handle.value for b in batches])
        self._h = ctypes.c_void_p()
        check(lib().bntt_multi_create(ctypes.byref(self._h), arr, len(batches)))

    def split(self, jobs) -> np.ndarray:
        owner = np.empty(len(jobs), dtype=np.uint32)
        check(lib().bntt_multi_split(self._h, jobs, len(jobs), owner.ctypes.data))
        return owner

    def run_host(self, jobs) -> None:
        check(lib().bntt_multi_run_host(self._h, jobs, len(jobs)))

    def close(self) -> None:
        if self._h:
            lib().bntt_multi_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The serving loop (bntt_server_*): continuous batching of NTT / vvmul /
    axpy requests on device-resident operands, admitted under an HBM budget."""

    def __init__(self, ctx: Context, plans: list[Plan], blas_q: int, blas_mu: int,
                 hbm_budget: int = 0, slots: int = 0, max_batch: int = 0):
        self.ctx, self.plans = ctx, plans
        self._blas = modulus(blas_q, blas_mu)
        cfg = ServerConfigC(hbm_budget, slots, max_batch)
        arr = (ctypes.c_void_p * len(plans))(*[p.handle.value for p in plans])
        self._h = ctypes.c_void_p()
        check(lib().bntt_server_create(ctx.handle, ctypes.byref(self._h), arr, len(plans),
                                       ctypes.byref(self._blas), ctypes.byref(cfg)))

    @property
    def handle(self):
        return self._h

    def clock(self) -> float:
        return lib().bntt_server_clock(self._h)

    def submit(self, req: RequestC) -> None:
        check(lib().bntt_server_submit(self._h, ctypes.byref(req)))

    def poll(self, cap: int = 1024) -> list:
        out = (CompletionC * cap)()
        n = ctypes.c_size_t()
        check(lib().bntt_server_poll(self._h, out, cap, ctypes.byref(n)))
        return [out[i] for i in range(n.value)]

    def release(self, y: int) -> None:
        check(lib().bntt_server_release(self._h, y))

    def drain(self) -> None:
        check(lib().bntt_server_drain(self._h))

    def stats(self) -> dict:
        st = ServerStatsC()
        check(lib().bntt_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStatsC._fields_}

    def replay(self, reqs, serial: bool = False, service: bool = False):
        """Latencies (s) of every request and the wall time of the replay;
        with service=True also each request's service time (completion less
        admission), as (latency, service, wall)."""
        n = len(reqs)
        lat = (ctypes.c_double * n)()
        svc = (ctypes.c_double * n)() if service else None
        wall = ctypes.c_double()
        check(lib().bntt_server_replay_ex(self._h, reqs, n, 1 if serial else 0, lat, svc,
                                          ctypes.byref(wall)))
        lat_a = np.frombuffer(lat, dtype=np.float64).copy()
        if service:
            return lat_a, np.frombuffer(svc, dtype=np.float64).copy(), wall.value
        return lat_a, wall.value

    def close(self) -> None:
        if self._h:
            lib().bntt_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------- BLAS helpers
def blas(ctx: Context, op: str, c, a, b, q: int, mu: int, x: int = 0,
         layout: int = LAYOUT_HILO) -> None:
    m = modulus(q, mu)
    L = lib()
    if _is_cuda_tensor(a):
        n = a.numel() // 2
        ptrs = (_dev_ptr(c), _dev_ptr(a), _dev_ptr(b))
        kind = "dev"
    else:
        n = a.size // 2
        ptrs = (_host_ptr(c), _host_ptr(a), _host_ptr(b))
        kind = "host"
    fn = getattr(L, f"bntt_{op}_{kind}")
    if op == "axpy":
        check(fn(ctx.handle, *ptrs, U128.of(x), n, ctypes.byref(m), layout))
    else:
        check(fn(ctx.handle, *ptrs, n, ctypes.byref(m), layout))


def fill_uniform(seed: int, count: int, q: int, offset: int = 0) -> np.ndarray:
    """Host-generated seeded residues in [0, q) (same values as the device fill)."""
    out = np.empty((count, 2), dtype=np.uint64)
    m = modulus(q, 0)
    check(lib().bntt_fill_uniform_host(_host_ptr(out), count, seed, offset, ctypes.byref(m),
                                       LAYOUT_HILO))
    return out


# ------------------------------------------- reference-shaped entry points
_DEFAULT_CTX: Context | None = None


def default_context() -> Context:
    global _DEFAULT_CTX
    if _DEFAULT_CTX is None:
        _DEFAULT_CTX = Context(0)
    return _DEFAULT_CTX


def ntt(Y: np.ndarray, X: np.ndarray, modulus_: int, mu: int, twiddles: np.ndarray) -> None:
    """Forward NTT of one input in place of the reference ntt()
    (src/ntt_scalar.c:582): N = len(X); Y receives the output."""
    X = pairs(X)
    n = X.shape[0]
    log2n = n.bit_length() - 1
    if n < 2 or (1 << log2n) != n:
        raise ValueError("N must be a power of two >= 2")
    plan = Plan(default_context(), log2n, modulus_, mu, twiddles)
    try:
        plan.forward(Y, X, 1)
    finally:
        plan.close()


def vector_add(c, a, b, m: int) -> None:
    blas(default_context(), "vvadd", c, pairs(a), pairs(b), m, 0)


def vector_sub(c, a, b, m: int) -> None:
    blas(default_context(), "vvsub", c, pairs(a), pairs(b), m, 0)


def vector_mul(c, a, b, m: int, mu: int) -> None:
    blas(default_context(), "vvmul", c, pairs(a), pairs(b), m, mu)


def axpy(c, a, b, x: int, m: int, mu: int) -> None:
    blas(default_context(), "axpy", c, pairs(a), pairs(b), m, mu, x)
