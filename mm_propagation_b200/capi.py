"""ctypes mirror of include/mmp.h and the loader for the native library.

The product's compute path is libmmp_b200.so (CUDA, sm_100a). This module only
declares the C structures and function signatures; it computes nothing. If the
library is missing, :func:`load` raises: there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libmmp_b200.so"
LIB_PATH = os.path.join(_HERE, LIB_NAME)

MMP_OK = 0
MMP_EINVAL = -1
MMP_ENOMEM = -2
MMP_ECUDA = -3
MMP_ENONFINITE = -4
MMP_ETIMEOUT = -5
MMP_ENOTSUP = -6
MMP_ENODEV = -7
MMP_ESTATE = -8
MMP_EDRIFT = -9

MMP_F_FP64 = 1 << 0
MMP_F_PHYSICAL_PAIRS = 1 << 1
MMP_F_CONTINUOUS = 1 << 2
MMP_F_NO_MONITORS = 1 << 3

MMP_RK_BY_ORDER = 0
MMP_RK_BUTCHER7_LAMBDA_MU = 1


class mmp_nz(C.Structure):
    _fields_ = [("p", C.c_uint32), ("k", C.c_uint32), ("l", C.c_uint32), ("m", C.c_uint32),
                ("value", C.c_double)]


class mmp_params(C.Structure):
    _fields_ = [
        ("n_modes", C.c_uint32),
        ("nt", C.c_uint32),
        ("n_beta", C.c_uint32),
        ("dispersion", C.POINTER(C.c_double)),
        ("n_nonzeros", C.c_uint32),
        ("coupling", C.POINTER(mmp_nz)),
        ("initial_fields", C.POINTER(C.c_double)),
        ("time_window", C.c_double),
        ("pulse_width", C.c_double),
        ("fiber_length", C.c_double),
        ("n_steps", C.c_uint32),
        ("method_order", C.c_uint32),
        ("nonlinearity_const", C.c_double),
        ("raman_proportion", C.c_double),
        ("raman_response", C.POINTER(C.c_double)),
        ("raman", C.c_int32),
        ("flags", C.c_uint32),
        ("rk_variant", C.c_int32),
        ("rk_lambda", C.c_double),
        ("rk_mu", C.c_double),
        ("center_frequency", C.c_double),
    ]


class mmp_info(C.Structure):
    _fields_ = [
        ("n_modes", C.c_uint32), ("nt", C.c_uint32), ("n_stages", C.c_uint32),
        ("n_pairs", C.c_uint32), ("n_pair_fields", C.c_uint32), ("pair_quirk_active", C.c_uint32),
        ("t_final", C.c_double), ("delta_t", C.c_double), ("z_final", C.c_double),
        ("delta_z", C.c_double), ("z", C.c_double),
        ("LD", C.c_double), ("conversion_factor", C.c_double), ("max_beta2", C.c_double),
        ("max_Q", C.c_double),
        ("steps_done", C.c_uint64),
        ("fp64", C.c_uint32),
        ("cluster_ctas", C.c_uint32),
        ("raman_recurrence", C.c_uint32),
        ("graph_branches", C.c_uint32),
        ("dense_contraction", C.c_uint32),
        ("tensor_core_contraction", C.c_uint32),
        ("contract_pair_chunk", C.c_uint32),
        ("contract_sub_block", C.c_uint32),
        ("contract_tile", C.c_uint32),
        ("autotuned", C.c_uint32),
    ]


class mmp_server_config(C.Structure):
    _fields_ = [
        ("memory_budget", C.c_uint64), ("max_slots", C.c_uint32),
        ("steps_per_tick", C.c_uint32), ("flags", C.c_uint32),
    ]


class mmp_request_info(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("n_modes", C.c_uint32), ("nt", C.c_uint32),
        ("steps", C.c_uint64),
        ("submit_s", C.c_double), ("start_s", C.c_double), ("done_s", C.c_double),
    ]


# name -> (restype, argtypes); every symbol include/mmp.h declares
SIGNATURES = {
    "mmp_validate_params": (C.c_int, [C.POINTER(mmp_params), C.c_char_p, C.c_size_t]),
    "mmp_solver_create": (C.c_int, [C.POINTER(mmp_params), C.POINTER(C.c_void_p)]),
    "mmp_propagate": (C.c_int, [C.c_void_p, C.c_uint32]),
    "mmp_propagate_async": (C.c_int, [C.c_void_p, C.c_uint32]),
    "mmp_synchronize": (C.c_int, [C.c_void_p]),
    "mmp_propagate_default": (C.c_int, [C.c_void_p]),
    "mmp_get_result": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "mmp_set_fields": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "mmp_get_monitors": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                   C.c_uint64, C.POINTER(C.c_uint64)]),
    "mmp_get_info": (C.c_int, [C.c_void_p, C.POINTER(mmp_info)]),
    "mmp_solver_destroy": (None, [C.c_void_p]),
    "mmp_batch_create": (C.c_int, [C.POINTER(C.POINTER(mmp_params)), C.c_uint32,
                                   C.POINTER(C.c_void_p)]),
    "mmp_batch_propagate": (C.c_int, [C.c_void_p, C.c_uint32]),
    "mmp_batch_propagate_async": (C.c_int, [C.c_void_p, C.c_uint32]),
    "mmp_batch_synchronize": (C.c_int, [C.c_void_p]),
    "mmp_batch_get_result": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]),
    "mmp_batch_set_fields": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]),
    "mmp_batch_get_info": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(mmp_info)]),
    "mmp_batch_size": (C.c_uint32, [C.c_void_p]),
    "mmp_batch_destroy": (None, [C.c_void_p]),
    "mmp_batch_propagate_timed": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_double)]),
    "mmp_batch_profile": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double),
                                    C.POINTER(C.c_uint32)]),
    "mmp_tableau": (C.c_int, [C.c_uint32, C.c_int32, C.c_double, C.c_double, C.POINTER(C.c_uint32),
                              C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "mmp_dft": (C.c_int, [C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.POINTER(C.c_double),
                         C.POINTER(C.c_double)]),
    "mmp_dft_noalloc": (C.c_int, [C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]),
    "mmp_propagate_snapshots": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int, C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "mmp_coupling_from_dense": (C.c_int, [C.c_uint32, C.POINTER(C.c_double), C.POINTER(mmp_nz),
                                          C.c_uint32, C.POINTER(C.c_uint32)]),
    "mmp_write_abs_text": (C.c_int, [C.c_char_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double)]),
    "mmp_write_mat": (C.c_int, [C.c_char_p, C.c_char_p, C.c_double, C.c_uint32, C.c_uint32,
                                C.POINTER(C.c_double), C.c_double]),
    "mmp_server_create":(C.c_int, [C.POINTER(mmp_server_config), C.POINTER(C.c_void_p)]),
    "mmp_server_submit": (C.c_int, [C.c_void_p, C.POINTER(mmp_params), C.POINTER(C.c_uint64)]),
    "mmp_server_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_int)]),
    "mmp_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.POINTER(C.c_double),
                                  C.POINTER(mmp_request_info)]),
    "mmp_server_destroy": (None, [C.c_void_p]),
    "mmp_strerror": (C.c_char_p, [C.c_int]),
    "mmp_last_error": (C.c_char_p, []),
    "mmp_version": (C.c_char_p, []),
    "mmp_kernel_launch_count": (C.c_uint64, []),
    "mmp_set_energy_drift_limit": (C.c_int, [C.c_void_p, C.c_double]),
    "mmp_batch_set_energy_drift_limit": (C.c_int, [C.c_void_p, C.c_uint32, C.c_double]),
    "mmp_debug_fail_alloc": (C.c_int, [C.c_int64]),
    "mmp_debug_live_allocations": (C.c_int64, []),
}

_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Load libmmp_b200.so (built by mm_propagation_b200/build.py) and bind
    every declared entry point. Raises OSError when the library is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError(f"{LIB_NAME} not built ({p} missing); run mm_propagation_b200/build.py")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
