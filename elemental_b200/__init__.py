"""elemental_b200 -- Python binding of libelemgpu.so (the sm_100a factor-and-solve kernels).

The product is the C ABI in include/elemgpu.h (and the C++ drop-in headers in
include/elemgpu/).  This module binds that ABI with ctypes for tests and
benchmarks: device-memory calls take column-major torch CUDA tensors, host
calls take column-major numpy arrays.  There is no CPU fallback: importing
raises if the CUDA library is missing, and every call raises if the library
reports an error.

Names follow Elemental (lapack-like/Cholesky.hpp, LU.hpp, HPDSolve.hpp,
GaussianElimination.hpp, blas-like/level3/{Trsm,Gemm,Herk}.hpp).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libelemgpu.so")

LOWER, UPPER = 0, 1
NORMAL, TRANSPOSE, ADJOINT = 0, 1, 2
LEFT, RIGHT = 0, 1
NON_UNIT, UNIT = 0, 1

OK, NOT_HPD, SINGULAR, TIMEOUT, NO_CONVERGENCE = 0, 1, 2, 3, 4


class ElemGPUError(RuntimeError):
    """A negative return code from libelemgpu (argument, CUDA or allocation error)."""


class NonHPDError(ValueError):
    """Cholesky met a non-positive pivot (the reference throws
    std::logic_error("A was not numerically HPD"), Cholesky/LVar3.hpp:37-38)."""

    def __init__(self, column):
        super().__init__(f"A was not numerically HPD (column {column})")
        self.column = column


class SingularMatrixError(ValueError):
    """LU met an exact zero pivot (SingularMatrixException, LU/Panel.hpp:76-77)."""

    def __init__(self, column):
        super().__init__(f"Matrix was singular (column {column})")
        self.column = column


class DeviceTimeoutError(RuntimeError):
    """A bounded device-side wait ran out; the kernel returned instead of hanging."""


_lib = None


def lib():
    """Load libelemgpu.so (build it first if a compiler is present)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _b
        _b.build()
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libelemgpu.so not found at {LIB_PATH}; run elemental_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    _declare(L)
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Names declared in include/elemgpu.h (used by the load/export test)."""
    import re
    hdr = open(os.path.join(_HERE, "..", "include", "elemgpu.h")).read()
    return re.findall(r"^EGPU_API [^()]*?\b(egpu_\w+)\(", hdr, flags=re.M)


def _declare(L):
    I, D, P, LL = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong
    H = ctypes.c_void_p
    sig = {
        "egpu_create": ([P, I], I),
        "egpu_destroy": ([H], I),
        "egpu_set_stream": ([H, P], I),
        "egpu_get_stream": ([H], P),
        "egpu_synchronize": ([H], I),
        "egpu_set_blocksize": ([H, I], I),
        "egpu_get_blocksize": ([H], I),
        "egpu_set_lookahead": ([H, I], I),
        "egpu_set_async": ([H, I], I),
        "egpu_get_status": ([H, P], I),
        "egpu_reserve": ([H, ctypes.c_size_t], I),
        "egpu_error_string": ([I], ctypes.c_char_p),
        "egpu_last_error_detail": ([], ctypes.c_char_p),
        "egpu_launch_count": ([H], LL),
        "egpu_trace_enable": ([H, I], I),
        "egpu_trace_summary": ([H, I, P, P, P, P], I),
        "egpu_trace_busy": ([H, I, P, P], I),
        "egpu_partition_systems": ([I, P, P, I, P, P], I),
        "egpu_sweep32_solve": ([H, I, I, I, P, I, P, I], I),
        "egpu_trace_events": ([H, I, P, P, P, P], I),
        "egpu_dpotrf": ([H, I, I, P, I, P], I),
        "egpu_dpotrs": ([H, I, I, I, I, P, I, P, I], I),
        "egpu_dposv": ([H, I, I, I, I, P, I, P, I, P], I),
        "egpu_dgetrf": ([H, I, I, P, I, P, P], I),
        "egpu_dgetrf_nopiv": ([H, I, I, P, I, P], I),
        "egpu_dgetrs": ([H, I, I, I, P, I, P, P, I], I),
        "egpu_dgesv": ([H, I, I, P, I, P, I, P], I),
        "egpu_dtrsm": ([H, I, I, I, I, I, I, D, P, I, P, I], I),
        "egpu_dtrsv": ([H, I, I, I, I, P, I, P], I),
        "egpu_dgemm": ([H, I, I, I, I, I, D, P, I, P, I, D, P, I], I),
        "egpu_dherk": ([H, I, I, I, I, D, P, I, D, P, I], I),
        "egpu_dlaswp": ([H, I, I, I, P, I, P, I], I),
        "egpu_dposv_batched": ([H, I, P, P, P, P, P, P, P], I),
        "egpu_dposv_mixed": ([H, I, I, I, P, I, P, I, P, I, I, D, P, P], I),
        "egpu_tc_gemm_split": ([H, I, I, I, D, P, I, P, I, D, P, I, I, I], I),
        "egpu_sweep32_queue": ([I, I, I, P, I], I),
        "egpu_host_dposv_mixed": ([H, I, I, I, P, I, P, I, P, I, I, D, P, P], I),
        "egpu_mixed_gmres_iterations": ([H], I),
        "egpu_set_mixed_policy": ([H, I], I),
        "egpu_dgesv_mixed": ([H, I, I, P, I, P, I, P, I, I, D, P, P], I),
        "egpu_mixed_mode": ([H], I),
        "egpu_mixed_condition_estimate": ([H, P], I),
        "egpu_batch_plan_create": ([H, I, I, P, P, P, P, P, P, P], I),
        "egpu_batch_plan_create_ex": ([H, I, I, I, P, P, P, P, P, P, P], I),
        "egpu_batch_plan_iters": ([P, P, P], I),
        "egpu_batch_plan_shape": ([P, P, P, P, P, P], I),
        "egpu_batch_plan_run": ([P, P], I),
        "egpu_batch_plan_info": ([P, P, P], I),
        "egpu_batch_plan_autotune": ([P, P, I, P, P], I),
        "egpu_batch_plan_set_grid": ([P, I], I),
        "egpu_batch_plan_destroy": ([P], I),
        "egpu_server_create": ([I, ctypes.c_size_t, I, I, P], I),
        "egpu_server_set_tolerance": ([P, D], I),
        "egpu_server_set_mixed_min_n": ([P, I], I),
        "egpu_server_submit": ([P, I, I, I, P, I, P, I, P, I, P], I),
        "egpu_server_register": ([P, I, I, P, I, P], I),
        "egpu_server_submit_resident": ([P, ctypes.c_ulonglong, I, P, I, P, I, P], I),
        "egpu_server_unregister": ([P, ctypes.c_ulonglong], I),
        "egpu_server_query": ([P, ctypes.c_ulonglong, I, P, P, P, P, P, P], I),
        "egpu_server_release": ([P, ctypes.c_ulonglong], I),
        "egpu_server_drain": ([P], I),
        "egpu_server_destroy": ([P], I),
        "egpu_dgesv_batched": ([H, I, P, P, P, P, P, P, P], I),
        "egpu_host_dpotrf": ([H, I, I, P, I, P], I),
        "egpu_host_dpotrs": ([H, I, I, I, I, P, I, P, I], I),
        "egpu_host_dposv": ([H, I, I, I, I, P, I, P, I, P], I),
        "egpu_host_dgetrf": ([H, I, I, P, I, P, P], I),
        "egpu_host_dgetrf_nopiv": ([H, I, I, P, I, P], I),
        "egpu_host_dgetrs": ([H, I, I, I, P, I, P, P, I], I),
        "egpu_host_dgesv": ([H, I, I, P, I, P, I, P], I),
        "egpu_host_dtrsm": ([H, I, I, I, I, I, I, D, P, I, P, I], I),
        "egpu_host_dgemm": ([H, I, I, I, I, I, D, P, I, P, I, D, P, I], I),
        "egpu_host_dherk": ([H, I, I, I, I, D, P, I, D, P, I], I),
        "egpu_host_dlaswp": ([H, I, I, I, P, I, P, I], I),
        "egpu_dldl": ([H, I, I, P, I, P, P], I),
        "egpu_host_dldl": ([H, I, I, P, I, P, P], I),
        "egpu_dpotrf_reverse": ([H, I, I, P, I, P], I),
        "egpu_host_dpotrf_reverse": ([H, I, I, P, I, P], I),
        "egpu_dtrtri": ([H, I, I, I, P, I], I),
        "egpu_dgetri": ([H, I, P, I, P], I),
        "egpu_dpotri": ([H, I, I, P, I, P], I),
        "egpu_dsafe_det": ([H, I, P, I, I, P, P], I),
        "egpu_dsafe_hpd_det": ([H, I, I, P, I, I, P, P], I),
        "egpu_host_dtrtri": ([H, I, I, I, P, I], I),
        "egpu_host_dgetri": ([H, I, P, I, P], I),
        "egpu_host_dpotri": ([H, I, I, P, I, P], I),
        "egpu_host_dsafe_det": ([H, I, P, I, I, P, P], I),
        "egpu_host_dsafe_hpd_det": ([H, I, I, P, I, I, P, P], I),
    }
    for name, (args, res) in sig.items():
        if hasattr(L, name):
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res


def _check(rc: int, info: int = 0):
    if rc == OK:
        return
    if rc == NOT_HPD:
        raise NonHPDError(info)
    if rc == SINGULAR:
        raise SingularMatrixError(info)
    if rc == TIMEOUT:
        raise DeviceTimeoutError(f"device wait timed out (site {info})")
    detail = lib().egpu_last_error_detail().decode()
    raise ElemGPUError(f"{lib().egpu_error_string(rc).decode()} ({rc}) {detail}")


# ------------------------------------------------------------ helpers --

def colmajor_cuda(a, device="cuda", dtype=None):
    """Copy a 2-D numpy/torch array into a column-major CUDA tensor (stride (1, rows))."""
    import torch
    t = torch.as_tensor(np.asarray(a) if not isinstance(a, torch.Tensor) else a)
    if dtype is not None:
        t = t.to(dtype)
    if t.dim() == 1:
        t = t.reshape(-1, 1)
    m, n = t.shape
    out = torch.empty_strided((m, n), (1, max(m, 1)), dtype=t.dtype, device=device)
    out.copy_(t)
    return out


def empty_colmajor(m, n, dtype=None, device="cuda", ld=None):
    import torch
    dtype = dtype or torch.float64
    ld = ld or max(m, 1)
    store = torch.empty(ld * max(n, 1), dtype=dtype, device=device)
    return torch.as_strided(store, (m, n), (1, ld))


def _ld(t) -> int:
    if t.dim() == 1:
        return max(t.shape[0], 1)
    if t.shape[1] <= 1:
        return max(t.shape[0], 1) if t.stride(0) == 1 else t.stride(1)
    if t.stride(0) != 1:
        raise ValueError("device matrices must be column-major (stride(0) == 1)")
    return t.stride(1)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _device_vec(t, count: int, dtype: str, device: int):
    """Pointer to a device-vector argument: a contiguous CUDA tensor of
    ``dtype`` ("int32" or "float64") on GPU ``device`` (the handle's) with at
    least ``count`` elements, the number the library reads or writes.  Checked
    here because a short, mistyped or other-GPU buffer would otherwise be
    written out of bounds (or through another device's pointer) by a kernel."""
    import torch
    want = {"int32": torch.int32, "float64": torch.float64}[dtype]
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
        raise TypeError(f"expected a CUDA tensor of {dtype}")
    if t.device.index != device:
        raise ValueError(f"expected a tensor on cuda:{device} (the handle's GPU), got {t.device}")
    if t.dtype != want:
        raise TypeError(f"expected a {dtype} tensor, got {t.dtype}")
    if not t.is_contiguous() or t.numel() < count:
        raise ValueError(f"expected a contiguous vector of at least {count} elements, got shape {tuple(t.shape)}")
    return ctypes.c_void_p(t.data_ptr())


def sweep32_queue(n: int, trans: int, sm_count: int = 148):
    """The tile-item queue the FP32 sweep launches for order n
    (egpu_sweep32_queue; host only): an int32 array of shape (items, 14) with
    columns map, dir, kind, nk, tm, tk, vrow, orow, orows, dep0, need0, dep1,
    need1, done."""
    import numpy as np
    cnt = lib().egpu_sweep32_queue(n, trans, sm_count, None, 0)
    _check(min(cnt, 0))
    out = np.zeros((max(cnt, 1), 14), dtype=np.int32)
    got = lib().egpu_sweep32_queue(n, trans, sm_count, out.ctypes.data_as(ctypes.c_void_p), cnt)
    _check(min(got, 0))
    return out[:cnt]


def partition_systems(n, kind, parts: int):
    """Owner part of each independent system (egpu_partition_systems): the
    systems are dealt largest first (cost n^3/3 HPD, 2n^3/3 GE) to the least
    loaded of `parts` parts.  Returns (owner int32 array, per-part load)."""
    n = np.ascontiguousarray(n, dtype=np.int32)
    k = None if kind is None else np.ascontiguousarray(kind, dtype=np.int32)
    owner = np.zeros(max(len(n), 1), dtype=np.int32)
    load = np.zeros(parts, dtype=np.float64)
    _check(lib().egpu_partition_systems(len(n), n.ctypes.data_as(ctypes.c_void_p),
                                        None if k is None else k.ctypes.data_as(ctypes.c_void_p), int(parts),
                                        owner.ctypes.data_as(ctypes.c_void_p), load.ctypes.data_as(ctypes.c_void_p)))
    return owner[:len(n)], load


def _np_f(a: np.ndarray):
    a = np.asarray(a)
    if a.dtype != np.float64:
        raise TypeError("host API expects float64 arrays")
    if a.ndim == 1:
        a = a.reshape(-1, 1, order="F")
    if not a.flags.f_contiguous:
        raise ValueError("host arrays must be Fortran-ordered (column-major)")
    return a


def _np_ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Server:
    """Continuous-batching request server (egpu_server_*).  Requests reference
    host arrays (column-major float64, best pinned) that must stay alive until
    the request completes."""

    HPD, GE = 0, 1

    def __init__(self, device=0, hbm_budget_bytes=150 << 30, slots=4, mode=0, tol=1e-14, mixed_min_n=None):
        self._s = ctypes.c_void_p()
        _check(lib().egpu_server_create(device, hbm_budget_bytes, slots, mode, ctypes.byref(self._s)))
        _check(lib().egpu_server_set_tolerance(self._s, tol))
        if mixed_min_n is not None:
            _check(lib().egpu_server_set_mixed_min_n(self._s, mixed_min_n))
        self._keep = {}

    def submit(self, kind, A, B, X):
        A, B, X = _np_f(A), _np_f(B), _np_f(X)
        rid = ctypes.c_ulonglong(0)
        _check(lib().egpu_server_submit(self._s, kind, A.shape[0], B.shape[1], _np_ptr(A), max(A.shape[0], 1),
                                        _np_ptr(B), max(B.shape[0], 1), _np_ptr(X), max(X.shape[0], 1),
                                        ctypes.byref(rid)))
        self._keep[rid.value] = (A, B, X)
        return rid.value

    def register(self, kind, A):
        """Copy A to the device once (resident); returns the matrix id for
        submit_resident.  The first request on it forms the factor, later ones
        reuse it."""
        A = _np_f(A)
        mid = ctypes.c_ulonglong(0)
        _check(lib().egpu_server_register(self._s, kind, A.shape[0], _np_ptr(A), max(A.shape[0], 1),
                                          ctypes.byref(mid)))
        return mid.value

    def submit_resident(self, mid, B, X):
        B, X = _np_f(B), _np_f(X)
        rid = ctypes.c_ulonglong(0)
        _check(lib().egpu_server_submit_resident(self._s, mid, B.shape[1], _np_ptr(B), max(B.shape[0], 1),
                                                 _np_ptr(X), max(X.shape[0], 1), ctypes.byref(rid)))
        self._keep[rid.value] = (B, X)
        return rid.value

    def unregister(self, mid):
        _check(lib().egpu_server_unregister(self._s, mid))

    def query(self, rid, wait=False):
        """None while pending, else a dict with status, latency_ms, path, iters, berr."""
        d, st, it, path = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        lat, be = ctypes.c_double(0.0), ctypes.c_double(0.0)
        _check(lib().egpu_server_query(self._s, rid, 1 if wait else 0, ctypes.byref(d), ctypes.byref(st),
                                       ctypes.byref(lat), ctypes.byref(path), ctypes.byref(it), ctypes.byref(be)))
        if not d.value:
            return None
        return {"status": st.value, "latency_ms": lat.value, "path": path.value, "iters": it.value,
                "berr": be.value}

    def release(self, rid):
        _check(lib().egpu_server_release(self._s, rid))
        self._keep.pop(rid, None)

    def drain(self):
        _check(lib().egpu_server_drain(self._s))

    def close(self):
        if self._s:
            lib().egpu_server_destroy(self._s)
            self._s = ctypes.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchPlan:
    """A device-resident batched solve (egpu_batch_plan_*): kind 0 = HPD solves,
    kind 1 = GaussianElimination.  The matrices stay where they are; run()
    only enqueues work (capturable in a CUDA graph).  precision 0: FP64 (each
    A receives its factor); precision 1: FP32 working copies + FP64 iterative
    refinement to backward error <= 1e-14 (the A are left unchanged)."""

    def __init__(self, handle, kind, As, Bs=None, precision=0):
        self.handle = handle
        cnt = len(As)
        n = (ctypes.c_int * cnt)(*[a.shape[0] for a in As])
        nr = (ctypes.c_int * cnt)(*[(b.shape[1] if b.dim() > 1 else 1) if Bs is not None else 0
                                    for b in (Bs if Bs is not None else As)])
        lda = (ctypes.c_int * cnt)(*[_ld(a) for a in As])
        ptrA = (ctypes.c_void_p * cnt)(*[a.data_ptr() for a in As])
        if Bs is not None:
            ldb = (ctypes.c_int * cnt)(*[_ld(b) for b in Bs])
            ptrB = (ctypes.c_void_p * cnt)(*[b.data_ptr() for b in Bs])
        else:
            ldb, ptrB = None, None
        self.count = cnt
        self._p = ctypes.c_void_p()
        self.precision = precision
        _check(lib().egpu_batch_plan_create_ex(handle._h, kind, precision, cnt, n, nr, ptrA, lda, ptrB, ldb,
                                               ctypes.byref(self._p)))

    @staticmethod
    def _stream(stream):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        return ctypes.c_void_p(s.cuda_stream or 1)  # 0 (legacy default stream) is passed as its handle 1

    def run(self, stream=None):
        _check(lib().egpu_batch_plan_run(self._p, self._stream(stream)))

    def info(self, stream=None):
        out = (ctypes.c_int * max(self.count, 1))()
        _check(lib().egpu_batch_plan_info(self._p, self._stream(stream), out))
        return list(out)[: self.count]

    def autotune(self, reps=2, stream=None):
        ms = ctypes.c_double(0.0)
        g = ctypes.c_int(0)
        _check(lib().egpu_batch_plan_autotune(self._p, self._stream(stream), reps, ctypes.byref(ms), ctypes.byref(g)))
        return ms.value, g.value

    def set_grid(self, grid):
        _check(lib().egpu_batch_plan_set_grid(self._p, grid))

    def iters(self, stream=None):
        """Refinement corrections per system of the last run (-1: the system
        was re-solved in FP64 after its refinement stalled; 0 for FP64 plans)."""
        out = (ctypes.c_int * max(self.count, 1))()
        _check(lib().egpu_batch_plan_iters(self._p, self._stream(stream), out))
        return list(out)[: self.count]

    def shape(self):
        """The launch shape per size class: [{"nmax", "panel", "threads", "grid"}]."""
        nc = ctypes.c_int(0)
        arr = [(ctypes.c_int * 3)() for _ in range(4)]
        _check(lib().egpu_batch_plan_shape(self._p, ctypes.byref(nc), *arr))
        return [{"nmax": arr[0][c], "panel": arr[1][c], "threads": arr[2][c], "grid": arr[3][c]}
                for c in range(nc.value)]

    def close(self):
        if self._p:
            lib().egpu_batch_plan_destroy(self._p)
            self._p = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Handle:
    """One egpu_context: stream + workspace on one device."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        _check(lib().egpu_create(ctypes.byref(h), device))
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().egpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def h(self):
        return self._h

    def _bind_stream(self):
        # Device-API calls run on torch's current stream so that they are
        # ordered after the torch ops that produced their inputs.
        import torch
        s = torch.cuda.current_stream(self.device).cuda_stream
        if s == 0:
            s = 1  # torch's default is the legacy stream (cudaStreamLegacy == 0x1)
        if s != getattr(self, "_bound", None):
            _check(lib().egpu_set_stream(self._h, ctypes.c_void_p(s)))
            self._bound = s

    def set_blocksize(self, nb: int):
        _check(lib().egpu_set_blocksize(self._h, nb))

    def blocksize(self) -> int:
        return lib().egpu_get_blocksize(self._h)

    def set_async(self, on: bool):
        """Device API only enqueues; failures are kept for get_status()."""
        _check(lib().egpu_set_async(self._h, int(on)))

    def get_status(self):
        """Wait for the handle's work; raise the first failure (and clear it)."""
        info = ctypes.c_int(0)
        _check(lib().egpu_get_status(self._h, ctypes.byref(info)), info.value)

    def reserve(self, nbytes: int):
        _check(lib().egpu_reserve(self._h, int(nbytes)))

    def set_lookahead(self, depth: int):
        """0: one stream, steps in order; 1: panel k+1 overlaps update k;
        G >= 2 (Cholesky): trailing updates deferred over groups of G panels,
        the side stream factoring each group's panels just in time; -1
        (default): G chosen per group from the trailing order."""
        _check(lib().egpu_set_lookahead(self._h, depth))

    def set_stream(self, stream_ptr: int | None):
        _check(lib().egpu_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)))
        self._bound = stream_ptr

    def synchronize(self):
        _check(lib().egpu_synchronize(self._h))

    def launch_count(self) -> int:
        return int(lib().egpu_launch_count(self._h))

    TRACE_KINDS = {"update": 0, "trsm": 1, "diag": 2, "panel": 3, "swap": 4, "other": 5, "tc": 6, "solve": 7}

    def trace_enable(self, on: bool = True):
        """Bracket every launch with CUDA events on its stream (clears old records)."""
        _check(lib().egpu_trace_enable(self._h, int(on)))

    def trace_events(self):
        """Traced launches in order: list of (kind name, stream, start ms, duration ms);
        stream 0 is the handle's stream, 1 the look-ahead side stream, 2 the
        lowest-priority auxiliary stream."""
        import numpy as np
        n = lib().egpu_trace_events(self._h, 0, None, None, None, None)
        if n < 0:
            _check(n)
        kinds = np.zeros(max(n, 1), dtype=np.int32)
        streams = np.zeros(max(n, 1), dtype=np.int32)
        st = np.zeros(max(n, 1), dtype=np.float64)
        du = np.zeros(max(n, 1), dtype=np.float64)
        lib().egpu_trace_events(self._h, n, kinds.ctypes.data_as(ctypes.c_void_p),
                                streams.ctypes.data_as(ctypes.c_void_p), st.ctypes.data_as(ctypes.c_void_p),
                                du.ctypes.data_as(ctypes.c_void_p))
        names = {v: k for k, v in self.TRACE_KINDS.items()}
        return [(names.get(int(kinds[i]), str(int(kinds[i]))), int(streams[i]), float(st[i]), float(du[i]))
                for i in range(n)]

    def trace_summary(self) -> dict:
        """{kind: {"ms", "flops", "bytes", "launches", "busy_ms", "share_ms"}} over
        the traced launches: "ms" sums per-launch durations; "busy_ms" is the
        union of the kind's launch intervals across streams; "share_ms" splits
        overlapped time evenly among the kinds in flight (the shares add up to
        the traced busy time)."""
        out = {}
        for name, k in self.TRACE_KINDS.items():
            ms, fl, by, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
            _check(lib().egpu_trace_summary(self._h, k, ctypes.byref(ms), ctypes.byref(fl), ctypes.byref(by),
                                            ctypes.byref(n)))
            busy, share = ctypes.c_double(), ctypes.c_double()
            _check(lib().egpu_trace_busy(self._h, k, ctypes.byref(busy), ctypes.byref(share)))
            out[name] = {"ms": ms.value, "flops": fl.value, "bytes": by.value, "launches": n.value,
                         "busy_ms": busy.value, "share_ms": share.value}
        return out

    def trace_busy_ms(self) -> float:
        """Busy time of the traced region (any kind in flight), ms."""
        busy = ctypes.c_double()
        _check(lib().egpu_trace_busy(self._h, -1, ctypes.byref(busy), None))
        return busy.value

    # ---------------- device API (torch CUDA tensors, column-major) ----
    def cholesky(self, A, uplo=LOWER):
        self._bind_stream()
        info = ctypes.c_int(0)
        rc = lib().egpu_dpotrf(self._h, uplo, A.shape[0], _ptr(A), _ld(A), ctypes.byref(info))
        _check(rc, info.value)

    def cholesky_solve_after(self, A, B, uplo=LOWER, orient=NORMAL):
        self._bind_stream()
        _check(lib().egpu_dpotrs(self._h, uplo, orient, A.shape[0], B.shape[1] if B.dim() > 1 else 1,
                                 _ptr(A), _ld(A), _ptr(B), _ld(B)))

    def hpd_solve(self, A, B, uplo=LOWER, orient=NORMAL):
        self._bind_stream()
        info = ctypes.c_int(0)
        rc = lib().egpu_dposv(self._h, uplo, orient, A.shape[0], B.shape[1] if B.dim() > 1 else 1,
                              _ptr(A), _ld(A), _ptr(B), _ld(B), ctypes.byref(info))
        _check(rc, info.value)

    def lu(self, A, p):
        self._bind_stream()
        info = ctypes.c_int(0)
        pp = _device_vec(p, min(A.shape[0], A.shape[1]), "int32", self.device)
        rc = lib().egpu_dgetrf(self._h, A.shape[0], A.shape[1], _ptr(A), _ld(A), pp, ctypes.byref(info))
        _check(rc, info.value)

    def ldl(self, A, d=None, orient=TRANSPOSE):
        """LDLT / LDLH(A[, d]): A = L D L^T without pivoting on the lower
        triangle (L strictly below the diagonal, D on it; d, a CUDA tensor of
        n doubles, also receives D)."""
        self._bind_stream()
        info = ctypes.c_int(0)
        dd = None if d is None else _device_vec(d, A.shape[0], "float64", self.device)
        rc = lib().egpu_dldl(self._h, orient, A.shape[0], _ptr(A), _ld(A), dd, ctypes.byref(info))
        _check(rc, info.value)

    def host_ldl(self, A: np.ndarray, orient=TRANSPOSE) -> np.ndarray:
        A = _np_f(A)
        d = np.zeros(A.shape[0])
        info = ctypes.c_int(0)
        rc = lib().egpu_host_dldl(self._h, orient, A.shape[0], _np_ptr(A), max(A.shape[0], 1), _np_ptr(d),
                                  ctypes.byref(info))
        _check(rc, info.value)
        return d

    def reverse_cholesky(self, A, uplo=LOWER):
        """ReverseCholesky(uplo, A): A = L^T L (LOWER) or U U^T (UPPER), in place."""
        self._bind_stream()
        info = ctypes.c_int(0)
        rc = lib().egpu_dpotrf_reverse(self._h, uplo, A.shape[0], _ptr(A), _ld(A), ctypes.byref(info))
        _check(rc, info.value)

    def host_reverse_cholesky(self, A: np.ndarray, uplo=LOWER):
        A = _np_f(A)
        info = ctypes.c_int(0)
        rc = lib().egpu_host_dpotrf_reverse(self._h, uplo, A.shape[0], _np_ptr(A), max(A.shape[0], 1),
                                            ctypes.byref(info))
        _check(rc, info.value)

    # ---- TriangularInverse / Inverse / HPDInverse / (Safe)Determinant ----

    def triangular_inverse(self, A, uplo=LOWER, diag=NON_UNIT):
        """TriangularInverse(uplo, diag, A) in place (the other triangle untouched)."""
        self._bind_stream()
        _check(lib().egpu_dtrtri(self._h, uplo, diag, A.shape[0], _ptr(A), _ld(A)))

    def inverse(self, A):
        """Inverse(A) in place via LU with partial pivoting."""
        self._bind_stream()
        info = ctypes.c_int(0)
        rc = lib().egpu_dgetri(self._h, A.shape[0], _ptr(A), _ld(A), ctypes.byref(info))
        _check(rc, info.value)

    def hpd_inverse(self, A, uplo=LOWER):
        """HPDInverse(uplo, A): the uplo triangle of A := that of inv(A)."""
        self._bind_stream()
        info = ctypes.c_int(0)
        rc = lib().egpu_dpotri(self._h, uplo, A.shape[0], _ptr(A), _ld(A), ctypes.byref(info))
        _check(rc, info.value)

    def safe_determinant(self, A, overwrite=False):
        """SafeDeterminant(A): (rho, kappa, n) with det(A) = rho * exp(kappa * n)."""
        self._bind_stream()
        rho, kappa = ctypes.c_double(0), ctypes.c_double(0)
        _check(lib().egpu_dsafe_det(self._h, A.shape[0], _ptr(A), _ld(A), int(bool(overwrite)),
                                    ctypes.byref(rho), ctypes.byref(kappa)))
        return rho.value, kappa.value, A.shape[0]

    def safe_hpd_determinant(self, A, uplo=LOWER, overwrite=False):
        """SafeHPDDeterminant(uplo, A): (rho, kappa, n), rho = 1 (0 if not HPD)."""
        self._bind_stream()
        rho, kappa = ctypes.c_double(0), ctypes.c_double(0)
        _check(lib().egpu_dsafe_hpd_det(self._h, uplo, A.shape[0], _ptr(A), _ld(A), int(bool(overwrite)),
                                        ctypes.byref(rho), ctypes.byref(kappa)))
        return rho.value, kappa.value, A.shape[0]

    def determinant(self, A):
        """Determinant(A) = rho * exp(kappa * n) (Determinant.hpp)."""
        rho, kappa, n = self.safe_determinant(A)
        return rho * float(np.exp(kappa * n))

    def hpd_determinant(self, A, uplo=LOWER):
        """HPDDeterminant(uplo, A) = exp(kappa * n)."""
        _, kappa, n = self.safe_hpd_determinant(A, uplo)
        return float(np.exp(kappa * n))

    def host_triangular_inverse(self, A: np.ndarray, uplo=LOWER, diag=NON_UNIT):
        A = _np_f(A)
        _check(lib().egpu_host_dtrtri(self._h, uplo, diag, A.shape[0], _np_ptr(A), max(A.shape[0], 1)))

    def host_inverse(self, A: np.ndarray):
        A = _np_f(A)
        info = ctypes.c_int(0)
        rc = lib().egpu_host_dgetri(self._h, A.shape[0], _np_ptr(A), max(A.shape[0], 1), ctypes.byref(info))
        _check(rc, info.value)

    def host_hpd_inverse(self, A: np.ndarray, uplo=LOWER):
        A = _np_f(A)
        info = ctypes.c_int(0)
        rc = lib().egpu_host_dpotri(self._h, uplo, A.shape[0], _np_ptr(A), max(A.shape[0], 1), ctypes.byref(info))
        _check(rc, info.value)

    def host_safe_determinant(self, A: np.ndarray, overwrite=False):
        A = _np_f(A)
        rho, kappa = ctypes.c_double(0), ctypes.c_double(0)
        _check(lib().egpu_host_dsafe_det(self._h, A.shape[0], _np_ptr(A), max(A.shape[0], 1), int(bool(overwrite)),
                                         ctypes.byref(rho), ctypes.byref(kappa)))
        return rho.value, kappa.value, A.shape[0]

    def host_safe_hpd_determinant(self, A: np.ndarray, uplo=LOWER, overwrite=False):
        A = _np_f(A)
        rho, kappa = ctypes.c_double(0), ctypes.c_double(0)
        _check(lib().egpu_host_dsafe_hpd_det(self._h, uplo, A.shape[0], _np_ptr(A), max(A.shape[0], 1),
                                             int(bool(overwrite)), ctypes.byref(rho), ctypes.byref(kappa)))
        return rho.value, kappa.value, A.shape[0]

    def lu_nopiv(self, A):
        self._bind_stream()
        info = ctypes.c_int(0)
        rc = lib().egpu_dgetrf_nopiv(self._h, A.shape[0], A.shape[1], _ptr(A), _ld(A), ctypes.byref(info))
        _check(rc, info.value)

    def lu_solve_after(self, A, p, B, orient=NORMAL):
        self._bind_stream()
        pp = None if p is None else _device_vec(p, A.shape[0], "int32", self.device)
        _check(lib().egpu_dgetrs(self._h, orient, A.shape[0], B.shape[1] if B.dim() > 1 else 1, _ptr(A), _ld(A),
                                 pp, _ptr(B), _ld(B)))

    def gaussian_elimination(self, A, B):
        self._bind_stream()
        info = ctypes.c_int(0)
        rc = lib().egpu_dgesv(self._h, A.shape[0], B.shape[1] if B.dim() > 1 else 1, _ptr(A), _ld(A), _ptr(B),
                              _ld(B), ctypes.byref(info))
        _check(rc, info.value)

    def trsm(self, side, uplo, orient, diag, alpha, A, B):
        self._bind_stream()
        m, n = B.shape[0], (B.shape[1] if B.dim() > 1 else 1)
        _check(lib().egpu_dtrsm(self._h, side, uplo, orient, diag, m, n, float(alpha), _ptr(A), _ld(A), _ptr(B),
                                _ld(B)))

    def trsv(self, uplo, orient, diag, A, x):
        self._bind_stream()
        _check(lib().egpu_dtrsv(self._h, uplo, orient, diag, A.shape[0], _ptr(A), _ld(A), _ptr(x)))

    def gemm(self, oA, oB, alpha, A, B, beta, C):
        self._bind_stream()
        m, n = C.shape
        k = A.shape[1] if oA == NORMAL else A.shape[0]
        _check(lib().egpu_dgemm(self._h, oA, oB, m, n, k, float(alpha), _ptr(A), _ld(A), _ptr(B), _ld(B),
                                float(beta), _ptr(C), _ld(C)))

    def herk(self, uplo, orient, alpha, A, beta, C):
        self._bind_stream()
        n = C.shape[0]
        k = A.shape[1] if orient == NORMAL else A.shape[0]
        _check(lib().egpu_dherk(self._h, uplo, orient, n, k, float(alpha), _ptr(A), _ld(A), float(beta), _ptr(C),
                                _ld(C)))

    def apply_row_pivots(self, B, p, inverse=False):
        self._bind_stream()
        m, n = B.shape[0], (B.shape[1] if B.dim() > 1 else 1)
        pp = _device_vec(p, p.shape[0], "int32", self.device)
        _check(lib().egpu_dlaswp(self._h, int(inverse), m, n, _ptr(B), _ld(B), pp, p.shape[0]))

    def _batched(self, fn, As, Bs):
        self._bind_stream()
        cnt = len(As)
        IA = ctypes.c_int * cnt
        PA = ctypes.c_void_p * cnt
        n = IA(*[a.shape[0] for a in As])
        lda = IA(*[_ld(a) for a in As])
        ptrA = PA(*[a.data_ptr() for a in As])
        if Bs is not None:
            nr = IA(*[(b.shape[1] if b.dim() > 1 else 1) for b in Bs])
            ldb = IA(*[_ld(b) for b in Bs])
            ptrB = PA(*[b.data_ptr() for b in Bs])
        else:
            nr = IA(*([0] * cnt))
            ldb = IA(*([1] * cnt))
            ptrB = None
        info = IA()
        _check(fn(self._h, cnt, n, nr, ptrA, lda, ptrB, ldb, info))
        return list(info)

    def gaussian_elimination_batched(self, As, Bs):
        """Batched GaussianElimination (LU with partial pivoting + solve), n <= 512,
        nrhs <= 16, one persistent launch.  Returns per-system info (0 or the
        1-based column of an exact zero pivot)."""
        return self._batched(lib().egpu_dgesv_batched, As, Bs)

    def hpd_solve_mixed(self, A, B, uplo=LOWER, max_iter=30, tol=1e-14):
        """Mixed-precision HPDSolve: returns (X, corrections, backward error).
        A and B (column-major float64 CUDA tensors) are left unchanged."""
        import torch
        self._bind_stream()
        nrhs = B.shape[1] if B.dim() > 1 else 1
        X = empty_colmajor(A.shape[0], nrhs, torch.float64, A.device)
        it = ctypes.c_int(0)
        be = ctypes.c_double(0.0)
        rc = lib().egpu_dposv_mixed(self._h, uplo, A.shape[0], nrhs, _ptr(A), _ld(A), _ptr(B), _ld(B), _ptr(X),
                                    _ld(X), max_iter, tol, ctypes.byref(it), ctypes.byref(be))
        if rc == NO_CONVERGENCE:
            raise ElemGPUError(f"refinement did not reach {tol:g} in {it.value} corrections (berr {be.value:.3e})")
        _check(rc)
        return X, it.value, be.value

    def gaussian_elimination_mixed(self, A, B, max_iter=30, tol=1e-14):
        """Mixed-precision GaussianElimination: returns (X, corrections,
        backward error); A and B (column-major float64 CUDA tensors) are left
        unchanged."""
        import torch
        self._bind_stream()
        nrhs = B.shape[1] if B.dim() > 1 else 1
        X = empty_colmajor(A.shape[0], nrhs, torch.float64, A.device)
        it = ctypes.c_int(0)
        be = ctypes.c_double(0.0)
        rc = lib().egpu_dgesv_mixed(self._h, A.shape[0], nrhs, _ptr(A), _ld(A), _ptr(B), _ld(B), _ptr(X), _ld(X),
                                    max_iter, tol, ctypes.byref(it), ctypes.byref(be))
        if rc == NO_CONVERGENCE:
            raise ElemGPUError(f"refinement did not reach {tol:g} in {it.value} corrections (berr {be.value:.3e})")
        if rc == SINGULAR:
            info = ctypes.c_int(0)
            lib().egpu_get_status(self._h, ctypes.byref(info))
            raise SingularMatrixError(info.value)
        _check(rc)
        return X, it.value, be.value

    def mixed_mode(self) -> int:
        """How the last mixed solve finished: 0 refinement, 1 GMRES-IR, 2 FP64 factors."""
        return int(lib().egpu_mixed_mode(self._h))

    def set_mixed_policy(self, policy: int):
        """0: adaptive (condition estimate only when refinement contracts
        slowly); 1: estimate after every factorization and pick IR or GMRES-IR."""
        _check(lib().egpu_set_mixed_policy(self._h, int(policy)))

    def mixed_condition_estimate(self) -> float:
        """kappa_1(A) estimated by the last mixed solve (-1 when it needed none)."""
        v = ctypes.c_double()
        _check(lib().egpu_mixed_condition_estimate(self._h, ctypes.byref(v)))
        return v.value

    def mixed_gmres_iterations(self):
        """GMRES iterations of the last mixed solve (0 when plain refinement converged)."""
        return lib().egpu_mixed_gmres_iterations(self._h)

    def sweep32_solve(self, L32, X, trans=0):
        """X := L^-1 X (trans 0), L^-T X (trans 1) or L^-T L^-1 X (trans 2) by the mixed solver's FP32
        super-block sweep (L: lower-triangular float32 CUDA tensor,
        column-major; X: float64, n x nrhs with nrhs <= 64)."""
        self._bind_stream()
        n = L32.shape[0]
        nrhs = X.shape[1] if X.dim() > 1 else 1
        ldl = L32.stride(1) if L32.dim() == 2 else max(n, 1)
        _check(lib().egpu_sweep32_solve(self._h, trans, n, nrhs, _ptr(L32), ldl, _ptr(X), _ld(X)))

    def tc_gemm_split(self, A, B, C, alpha=1.0, beta=0.0, lower=False, terms=3):
        """C (float32, column-major) = alpha A B^T + beta C on the tcgen05 tensor cores
        (A, B float64 column-major, split into TF32 hi/lo parts)."""
        self._bind_stream()
        _check(lib().egpu_tc_gemm_split(self._h, A.shape[0], B.shape[0], A.shape[1], alpha, _ptr(A), _ld(A), _ptr(B),
                                        _ld(B), beta, _ptr(C), _ld(C), 1 if lower else 0, terms))

    def hpd_solve_batched(self, As, Bs=None):
        """Batched HPDSolve(LOWER) over lists of column-major CUDA tensors (n <= 512,
        nrhs <= 16) in one persistent launch.  Returns the per-system info list
        (0, or the 1-based column where that system stopped being HPD)."""
        self._bind_stream()
        cnt = len(As)
        IA = ctypes.c_int * cnt
        PA = ctypes.c_void_p * cnt
        n = IA(*[a.shape[0] for a in As])
        lda = IA(*[_ld(a) for a in As])
        ptrA = PA(*[a.data_ptr() for a in As])
        if Bs is not None:
            nr = IA(*[(b.shape[1] if b.dim() > 1 else 1) for b in Bs])
            ldb = IA(*[_ld(b) for b in Bs])
            ptrB = PA(*[b.data_ptr() for b in Bs])
        else:
            nr = IA(*([0] * cnt))
            ldb = IA(*([1] * cnt))
            ptrB = None
        info = IA()
        _check(lib().egpu_dposv_batched(self._h, cnt, n, nr, ptrA, lda, ptrB, ldb, info))
        return list(info)

    # ---------------- host API (numpy, Fortran order, in place) --------
    def host_cholesky(self, A: np.ndarray, uplo=LOWER):
        A = _np_f(A)
        info = ctypes.c_int(0)
        rc = lib().egpu_host_dpotrf(self._h, uplo, A.shape[0], _np_ptr(A), max(A.shape[0], 1), ctypes.byref(info))
        _check(rc, info.value)

    def host_hpd_solve(self, A: np.ndarray, B: np.ndarray, uplo=LOWER, orient=NORMAL):
        A, B = _np_f(A), _np_f(B)
        info = ctypes.c_int(0)
        rc = lib().egpu_host_dposv(self._h, uplo, orient, A.shape[0], B.shape[1], _np_ptr(A), max(A.shape[0], 1),
                                   _np_ptr(B), max(B.shape[0], 1), ctypes.byref(info))
        _check(rc, info.value)

    def host_cholesky_solve_after(self, A, B, uplo=LOWER, orient=NORMAL):
        A, B = _np_f(A), _np_f(B)
        _check(lib().egpu_host_dpotrs(self._h, uplo, orient, A.shape[0], B.shape[1], _np_ptr(A),
                                      max(A.shape[0], 1), _np_ptr(B), max(B.shape[0], 1)))

    def host_lu(self, A: np.ndarray) -> np.ndarray:
        A = _np_f(A)
        m, n = A.shape
        p = np.zeros(min(m, n), dtype=np.int32)
        info = ctypes.c_int(0)
        rc = lib().egpu_host_dgetrf(self._h, m, n, _np_ptr(A), max(m, 1), _np_ptr(p), ctypes.byref(info))
        _check(rc, info.value)
        return p

    def host_lu_nopiv(self, A: np.ndarray):
        A = _np_f(A)
        info = ctypes.c_int(0)
        rc = lib().egpu_host_dgetrf_nopiv(self._h, A.shape[0], A.shape[1], _np_ptr(A), max(A.shape[0], 1),
                                          ctypes.byref(info))
        _check(rc, info.value)

    def host_lu_solve_after(self, A, p, B, orient=NORMAL):
        A, B = _np_f(A), _np_f(B)
        pp = None if p is None else np.ascontiguousarray(p, dtype=np.int32)
        _check(lib().egpu_host_dgetrs(self._h, orient, A.shape[0], B.shape[1], _np_ptr(A), max(A.shape[0], 1),
                                      None if pp is None else _np_ptr(pp), _np_ptr(B), max(B.shape[0], 1)))

    def host_hpd_solve_mixed(self, A, B, X, uplo=LOWER, max_iter=30, tol=1e-14):
        """Mixed-precision HPD solve on host arrays: X := A^-1 B (A, B unchanged);
        returns (corrections, backward error)."""
        A, B, X = _np_f(A), _np_f(B), _np_f(X)
        it = ctypes.c_int(0)
        be = ctypes.c_double(0.0)
        rc = lib().egpu_host_dposv_mixed(self._h, uplo, A.shape[0], B.shape[1], _np_ptr(A), max(A.shape[0], 1),
                                         _np_ptr(B), max(B.shape[0], 1), _np_ptr(X), max(X.shape[0], 1), max_iter,
                                         tol, ctypes.byref(it), ctypes.byref(be))
        if rc == NO_CONVERGENCE:
            raise ElemGPUError(f"refinement did not reach {tol:g} in {it.value} corrections (berr {be.value:.3e})")
        _check(rc)
        return it.value, be.value

    def host_gaussian_elimination(self, A, B):
        A, B = _np_f(A), _np_f(B)
        info = ctypes.c_int(0)
        rc = lib().egpu_host_dgesv(self._h, A.shape[0], B.shape[1], _np_ptr(A), max(A.shape[0], 1), _np_ptr(B),
                                   max(B.shape[0], 1), ctypes.byref(info))
        _check(rc, info.value)

    def host_trsm(self, side, uplo, orient, diag, alpha, A, B):
        A, B = _np_f(A), _np_f(B)
        _check(lib().egpu_host_dtrsm(self._h, side, uplo, orient, diag, B.shape[0], B.shape[1], float(alpha),
                                     _np_ptr(A), max(A.shape[0], 1), _np_ptr(B), max(B.shape[0], 1)))

    def host_gemm(self, oA, oB, alpha, A, B, beta, C):
        A, B, C = _np_f(A), _np_f(B), _np_f(C)
        m, n = C.shape
        k = A.shape[1] if oA == NORMAL else A.shape[0]
        _check(lib().egpu_host_dgemm(self._h, oA, oB, m, n, k, float(alpha), _np_ptr(A), max(A.shape[0], 1),
                                     _np_ptr(B), max(B.shape[0], 1), float(beta), _np_ptr(C), max(m, 1)))

    def host_herk(self, uplo, orient, alpha, A, beta, C):
        A, C = _np_f(A), _np_f(C)
        n = C.shape[0]
        k = A.shape[1] if orient == NORMAL else A.shape[0]
        _check(lib().egpu_host_dherk(self._h, uplo, orient, n, k, float(alpha), _np_ptr(A), max(A.shape[0], 1),
                                     float(beta), _np_ptr(C), max(n, 1)))

    def host_apply_row_pivots(self, B, p, inverse=False):
        B = _np_f(B)
        pp = np.ascontiguousarray(p, dtype=np.int32)
        _check(lib().egpu_host_dlaswp(self._h, int(inverse), B.shape[0], B.shape[1], _np_ptr(B),
                                      max(B.shape[0], 1), _np_ptr(pp), len(pp)))
