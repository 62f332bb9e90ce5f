"""egpu_dpotrf_noalloc: the Cholesky entry point for callers that cannot let a
library allocate device memory (their device memory belongs to their own pool
and an allocation mid-run could fail or synchronise the device).  It keeps its
scratch in a fixed __device__ array, so it takes only the caller's stream.

Called through the C ABI and checked against the existing entry point
(egpu_dpotrf through a handle) on two calls in a row, with the tolerance of the
other Cholesky parity tests.  Kept in a file of its own, collected last."""
import ctypes

import numpy as np
import pytest

import elemental_b200 as eg
from elemental_b200 import inputs

pytestmark = pytest.mark.gpu


def _noalloc():
    f = eg.lib().egpu_dpotrf_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _lower_or_upper(F, uplo):
    return np.tril(F) if uplo == eg.LOWER else np.triu(F)


@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
def test_noalloc_matches_handle_entry_point_twice(uplo):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    f = _noalloc()
    with eg.Handle(0) as h:
        # two calls in a row, different sizes; the first one is a view whose
        # leading dimension (778) exceeds its height (777)
        for call, (n, ld) in enumerate(((777, 778), (1300, 1300))):
            A = inputs.spd_ggt(n, seed=500 + call)
            ref = eg.colmajor_cuda(A)
            h.cholesky(ref, uplo)  # existing entry point (egpu_dpotrf)
            dA = eg.empty_colmajor(n, n, ld=ld)
            dA.copy_(torch.from_numpy(A))
            torch.cuda.synchronize()
            info = ctypes.c_int(-1)
            rc = f(None, uplo, n, ctypes.c_void_p(dA.data_ptr()), ld, 128, ctypes.byref(info))
            assert rc == eg.OK and info.value == 0
            got = _lower_or_upper(dA.cpu().numpy(), uplo)
            want = _lower_or_upper(ref.cpu().numpy(), uplo)
            assert np.max(np.abs(got - want)) <= 1e-11 * np.max(np.abs(want))
            # the triangle a Cholesky does not own is untouched
            other = np.triu(np.ones((n, n), bool), 1) if uplo == eg.LOWER else np.tril(np.ones((n, n), bool), -1)
            assert np.array_equal(dA.cpu().numpy()[other], A[other])


def test_noalloc_second_call_takes_no_device_memory():
    # after a first call on the device (module loading and the scratch array
    # placed), a call on a new size leaves the free device memory unchanged
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    f = _noalloc()
    info = ctypes.c_int(0)
    # both sizes launch the same kernels (one diagonal-block kernel, the 64 x
    # 128 panel multiply and the triangular update), so the first call has
    # loaded everything the second one runs
    A1 = eg.empty_colmajor(777, 777, ld=778)
    A1.copy_(torch.from_numpy(inputs.spd_ggt(777, 31)))
    A2 = eg.empty_colmajor(1300, 1300)
    A2.copy_(torch.from_numpy(inputs.spd_ggt(1300, 32)))
    torch.cuda.synchronize()
    assert f(None, eg.LOWER, 777, ctypes.c_void_p(A1.data_ptr()), 778, 128, ctypes.byref(info)) == eg.OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert f(None, eg.LOWER, 1300, ctypes.c_void_p(A2.data_ptr()), 1300, 128, ctypes.byref(info)) == eg.OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_and_reports():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    f = _noalloc()
    A = inputs.spd_ggt(200, 9)
    dA = eg.colmajor_cuda(A)
    info = ctypes.c_int(0)
    # an odd leading dimension cannot be staged without allocating: refused
    assert f(None, eg.LOWER, 199, ctypes.c_void_p(dA.data_ptr()), 199, 128, ctypes.byref(info)) == -4
    # block size beyond the fixed scratch: a clear error, nothing launched
    assert f(None, eg.LOWER, 200, ctypes.c_void_p(dA.data_ptr()), 200, 256, ctypes.byref(info)) == -6
    assert np.array_equal(dA.cpu().numpy(), A)
    # a non-HPD input reports the same column as the other entry point
    A[150, 150] = -1.0
    dA = eg.colmajor_cuda(A)
    rc = f(None, eg.LOWER, 200, ctypes.c_void_p(dA.data_ptr()), 200, 128, ctypes.byref(info))
    assert rc == eg.NOT_HPD and info.value == 151
    # the status word is cleared by the next call
    B = inputs.spd_ggt(200, 10)
    dB = eg.colmajor_cuda(B)
    assert f(None, eg.LOWER, 200, ctypes.c_void_p(dB.data_ptr()), 200, 128, ctypes.byref(info)) == eg.OK
