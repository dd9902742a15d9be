"""mmp_dft_noalloc: the transform for callers that must not allocate device memory
(their pool belongs to another allocator, or they cannot take the synchronisation
of cudaMalloc/cudaFree). It must give the same results as mmp_dft, call after call,
out of its static staging buffer, and a call after the first must take no device
memory. This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from mm_propagation_b200 import capi

pytestmark = pytest.mark.gpu


def _noalloc(x, inverse, fp64):
    lib = capi.load()
    a = np.ascontiguousarray(np.atleast_2d(x), dtype=np.complex128)
    out = np.empty_like(a)
    rows, n = a.shape
    rc = lib.mmp_dft_noalloc(n, rows, 1 if inverse else -1, 1 if fp64 else 0,
                             a.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                             out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
    return rc, out


CASES = [(4096, 5, True), (16384, 3, False), (65536, 2, True), (32768, 4, False), (256, 64, True)]


def _free_device_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_noalloc_matches_dft_two_calls_in_a_row(mmp):
    rng = np.random.default_rng(7)
    inputs, refs = [], []
    for n, rows, fp64 in CASES:  # every reference result first: mmp_dft allocates
        for inverse in (False, True):
            x = rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))
            inputs.append((x, inverse, fp64))
            refs.append(mmp.dft(x, inverse=inverse, fp64=fp64))
    lib = capi.load()
    free = []
    for call in range(2):  # the second pass reuses the buffer the first one left behind
        free.append(_free_device_bytes())
        l0 = lib.mmp_kernel_launch_count()
        for (x, inverse, fp64), ref in zip(inputs, refs):
            rc, got = _noalloc(x, inverse, fp64)
            assert rc == 0, (call, x.shape, fp64, inverse, rc, capi.load().mmp_last_error())
            tol = 1e-13 if fp64 else 2e-6
            err = np.abs(got - ref).max() / np.abs(ref).max()
            assert err < tol, (call, x.shape, fp64, inverse, err)
        # one transform launch per call (the first call on a device also fills its tables)
        assert lib.mmp_kernel_launch_count() - l0 >= len(inputs)
    free.append(_free_device_bytes())
    # after the first pass (set-up, lazily loaded kernels) no call takes device memory
    assert free[2] == free[1], free


def test_noalloc_rejects_oversize(mmp):
    x = np.zeros((17, 65536), dtype=np.complex128)  # 17 * 2^16 > 2^20 samples
    rc, _ = _noalloc(x, False, True)
    assert rc == capi.MMP_EINVAL
    assert b"2^20" in capi.load().mmp_last_error()
