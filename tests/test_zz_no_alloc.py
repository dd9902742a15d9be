"""mmp_dft_noalloc: the transform for callers that must not allocate device memory
(their pool belongs to another allocator, or they cannot take the synchronisation
of cudaMalloc/cudaFree). It must give the same results as mmp_dft, call after call,
out of its static staging buffer. This file is collected last on purpose."""
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


def test_noalloc_matches_dft_two_calls_in_a_row(mmp):
    rng = np.random.default_rng(7)
    for call in range(2):  # the second call reuses the buffer the first one left behind
        for n, rows, fp64 in CASES:
            for inverse in (False, True):
                x = rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))
                ref = mmp.dft(x, inverse=inverse, fp64=fp64)
                rc, got = _noalloc(x, inverse, fp64)
                assert rc == 0, (call, n, rows, fp64, inverse, rc)
                tol = 1e-13 if fp64 else 2e-6
                err = np.abs(got - ref).max() / np.abs(ref).max()
                assert err < tol, (call, n, rows, fp64, inverse, err)


def test_noalloc_rejects_oversize(mmp):
    x = np.zeros((17, 65536), dtype=np.complex128)  # 17 * 2^16 > 2^20 samples
    rc, _ = _noalloc(x, False, True)
    assert rc == capi.MMP_EINVAL
