"""ctypes loader for oracle/_ref/libmmref.so — the reference's own CPU solver.

TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT (see oracle/mmp_oracle.py). The
library is built from the unmodified reference sources by oracle/Makefile; this
module only calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(_HERE, "_ref", "libmmref.so")
sys.path.insert(0, os.path.dirname(_HERE))
from mm_propagation_b200 import capi  # noqa: E402  (ctypes struct layout only)

NO_ARG = 0xFFFFFFFF  # chunk value meaning computeLawsonRK() without argument

_lib = None


def available() -> bool:
    return os.path.exists(REF_LIB)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not available():
            raise OSError(f"{REF_LIB} missing: run `make -C oracle`")
        _lib = C.CDLL(REF_LIB)
        _lib.mmref_run.restype = C.c_int
        _lib.mmref_run.argtypes = [C.POINTER(capi.mmp_params), C.POINTER(C.c_uint), C.c_uint,
                                   C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib.mmref_fft.restype = C.c_int
        _lib.mmref_fft.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib.mmref_initial_threads.restype = C.c_int
        _lib.mmref_effective_threads.restype = C.c_int
        _lib.mmref_effective_threads.argtypes = [C.c_uint]
    return _lib


def run(prob, chunks=None):
    """Reference solve: computeLawsonRK(c) for each chunk (default [n_steps]; None
    entries mean the no-argument form), then getResult(). Returns
    (phi complex128 [M][NT], seconds of compute)."""
    chunks = [prob.n_steps] if chunks is None else [NO_ARG if c is None else int(c) for c in chunks]
    h = prob.to_params()
    arr = (C.c_uint * len(chunks))(*chunks)
    out = np.zeros((prob.n_modes, prob.nt), dtype=np.complex128)
    sec = C.c_double(0.0)
    rc = lib().mmref_run(h.ptr(), arr, len(chunks),
                         out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)), C.byref(sec))
    if rc != 0:
        raise RuntimeError(f"mmref_run failed ({rc})")
    return out, sec.value


def fft(x, sign=-1):
    """The FFTW-API shim's transform (unnormalised)."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.zeros_like(x)
    lib().mmref_fft(len(x), sign, x.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                    out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
    return out


def threads(M: int):
    return lib().mmref_initial_threads(), lib().mmref_effective_threads(M)
