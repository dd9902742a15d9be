"""mm_propagation_b200 — Lawson–Runge–Kutta multimode NLSE solver on B200 (sm_100a).

Python face of the C ABI in include/mmp.h (the C++ drop-in classes live in
include/MultimodePropagation_B200.hpp). Every computation runs in
libmmp_b200.so's CUDA kernels; if the library or a B200 is missing, calls
raise. There is no CPU fallback.

    from mm_propagation_b200 import Solver, workloads
    prob = workloads.grin2(peak_scale=0.01)
    with Solver(prob) as s:
        s.propagate(prob.n_steps)      # computeLawsonRK(n_steps)
        phi = s.result()               # getResult(), complex128 [M][NT]
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import capi, workloads  # noqa: F401
from .capi import (MMP_F_CONTINUOUS, MMP_F_FP64, MMP_F_NO_MONITORS,  # noqa: F401
                   MMP_F_PHYSICAL_PAIRS, MMP_RK_BUTCHER7_LAMBDA_MU, MMP_RK_BY_ORDER)

__all__ = ["Solver", "Batch", "Server", "MMPError", "dft", "lib", "workloads", "capi"]


class MMPError(RuntimeError):
    def __init__(self, code: int, where: str):
        l = capi.load()
        detail = l.mmp_last_error().decode()
        super().__init__(f"{where}: {l.mmp_strerror(code).decode()} ({code}): {detail}")
        self.code = code


def lib() -> C.CDLL:
    return capi.load()


def _check(rc: int, where: str):
    if rc != 0:
        raise MMPError(rc, where)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def validate(prob) -> tuple[int, str]:
    h = prob.to_params()
    buf = C.create_string_buffer(512)
    rc = lib().mmp_validate_params(h.ptr(), buf, 512)
    return rc, buf.value.decode()


def tableau(method_order: int = 4, rk_variant: int = 0, lam: float = 0.0, mu: float = 0.0):
    """(a, b, c) of the RK tableau the solver uses for these settings (host-side data)."""
    s = C.c_uint32(0)
    a = (C.c_double * 121)()
    b = (C.c_double * 11)()
    c = (C.c_double * 11)()
    _check(lib().mmp_tableau(method_order, rk_variant, lam, mu, C.byref(s), a, b, c), "mmp_tableau")
    n = s.value
    return ([[a[i * 11 + j] for j in range(i)] for i in range(n)], list(b[:n]), list(c[:n]))


def info_dict(info: capi.mmp_info) -> dict:
    return {name: getattr(info, name) for name, _ in info._fields_}


class Solver:
    """One solve: MultimodePropagationB200_RamanOFF/ON behind the C ABI."""

    def __init__(self, prob):
        self.prob = prob
        self._h = prob.to_params()
        self._ptr = C.c_void_p()
        _check(lib().mmp_solver_create(self._h.ptr(), C.byref(self._ptr)), "mmp_solver_create")
        self.M, self.nt = prob.n_modes, prob.nt

    def propagate(self, nz: int | None = None):
        """computeLawsonRK(nz); nz=None means computeLawsonRK() (floor(z_final/dz) steps)."""
        if nz is None:
            _check(lib().mmp_propagate_default(self._ptr), "mmp_propagate_default")
        else:
            _check(lib().mmp_propagate(self._ptr, int(nz)), "mmp_propagate")

    def propagate_async(self, nz: int):
        _check(lib().mmp_propagate_async(self._ptr, int(nz)), "mmp_propagate_async")

    def synchronize(self):
        _check(lib().mmp_synchronize(self._ptr), "mmp_synchronize")

    def result(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.M, self.nt), dtype=np.complex128)
        _check(lib().mmp_get_result(self._ptr, _dptr(out.view(np.float64))), "mmp_get_result")
        return out

    def set_fields(self, phi0: np.ndarray):
        a = np.ascontiguousarray(phi0, dtype=np.complex128)
        _check(lib().mmp_set_fields(self._ptr, _dptr(a.view(np.float64))), "mmp_set_fields")

    def snapshots(self, n_save: int, z_mode: int = 0):
        """The MEX front end's chunked run (mmp_propagate_snapshots): returns
        (fields complex128 [n_save][M][NT], Z [n_save] in m, elapsed [n_save] in s).
        z_mode 0 carries z across chunks; 1 restarts it per chunk as the reference does."""
        f = np.empty((n_save, self.M, self.nt), dtype=np.complex128)
        z = np.empty(n_save)
        t = np.empty(n_save)
        _check(lib().mmp_propagate_snapshots(self._ptr, int(n_save), int(z_mode), _dptr(f.view(np.float64)),
                                             _dptr(z), _dptr(t)), "mmp_propagate_snapshots")
        return f, z, t

    def monitors(self, max_steps: int | None = None):
        info = self.info()
        n = info["steps_done"] if max_steps is None else max_steps
        e = np.zeros(max(n, 1))
        p = np.zeros(max(n, 1))
        w = C.c_uint64(0)
        _check(lib().mmp_get_monitors(self._ptr, _dptr(e), _dptr(p), n, C.byref(w)), "mmp_get_monitors")
        return e[:w.value], p[:w.value]

    def info(self) -> dict:
        i = capi.mmp_info()
        _check(lib().mmp_get_info(self._ptr, C.byref(i)), "mmp_get_info")
        return info_dict(i)

    def set_energy_drift_limit(self, rel_tol: float):
        """Fail later propagate calls with MMP_EDRIFT once the FP64 energy monitor moves by
        more than rel_tol of the first step's energy (0 turns the check off)."""
        _check(lib().mmp_set_energy_drift_limit(self._ptr, float(rel_tol)), "mmp_set_energy_drift_limit")

    def close(self):
        if self._ptr:
            lib().mmp_solver_destroy(self._ptr)
            self._ptr = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent solves advanced together by the same launches (shared NT,
    precision, Raman choice and RK tableau)."""

    def __init__(self, probs):
        self.probs = list(probs)
        self._hs = [p.to_params() for p in self.probs]
        arr = (C.POINTER(capi.mmp_params) * len(self._hs))(*[h.ptr() for h in self._hs])
        self._ptr = C.c_void_p()
        _check(lib().mmp_batch_create(arr, len(self._hs), C.byref(self._ptr)), "mmp_batch_create")

    def __len__(self):
        return len(self.probs)

    def propagate(self, nz: int):
        _check(lib().mmp_batch_propagate(self._ptr, int(nz)), "mmp_batch_propagate")

    def propagate_async(self, nz: int):
        _check(lib().mmp_batch_propagate_async(self._ptr, int(nz)), "mmp_batch_propagate_async")

    def synchronize(self):
        _check(lib().mmp_batch_synchronize(self._ptr), "mmp_batch_synchronize")

    def propagate_timed(self, nz: int, repeats: int = 1) -> float:
        """repeats x propagate(nz) timed with CUDA events on the batch's stream (ms)."""
        ms = C.c_double(0.0)
        _check(lib().mmp_batch_propagate_timed(self._ptr, int(nz), int(repeats), C.byref(ms)),
               "mmp_batch_propagate_timed")
        return ms.value

    def profile(self, nz: int) -> dict:
        """Per-kernel mean device time of one launch (ms) over nz un-graphed steps."""
        ms = (C.c_double * 3)()
        n = (C.c_uint32 * 3)()
        _check(lib().mmp_batch_profile(self._ptr, int(nz), ms, n), "mmp_batch_profile")
        return {k: {"ms_per_launch": ms[i], "launches": n[i]}
                for i, k in enumerate(("pair", "contract", "nu"))}

    def result(self, i: int, out: np.ndarray | None = None) -> np.ndarray:
        p = self.probs[i]
        if out is None:
            out = np.empty((p.n_modes, p.nt), dtype=np.complex128)
        _check(lib().mmp_batch_get_result(self._ptr, i, _dptr(out.view(np.float64))), "mmp_batch_get_result")
        return out

    def set_fields(self, i: int, phi0: np.ndarray):
        a = np.ascontiguousarray(phi0, dtype=np.complex128)
        _check(lib().mmp_batch_set_fields(self._ptr, i, _dptr(a.view(np.float64))), "mmp_batch_set_fields")

    def info(self, i: int) -> dict:
        inf = capi.mmp_info()
        _check(lib().mmp_batch_get_info(self._ptr, i, C.byref(inf)), "mmp_batch_get_info")
        return info_dict(inf)

    def set_energy_drift_limit(self, i: int, rel_tol: float):
        _check(lib().mmp_batch_set_energy_drift_limit(self._ptr, i, float(rel_tol)),
               "mmp_batch_set_energy_drift_limit")

    def close(self):
        if self._ptr:
            lib().mmp_batch_destroy(self._ptr)
            self._ptr = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request loop with continuous batching: submit whole solves (each runs its own
    n_steps from its initial fields); a device worker admits them into slot pools of
    their kernel shape as memory allows, advances every pool steps_per_tick steps per
    replay and retires finished solves. Results equal a standalone Solver's."""

    def __init__(self, memory_budget: int = 0, max_slots: int = 0, steps_per_tick: int = 0,
                 flags: int = 0):
        cfg = capi.mmp_server_config(memory_budget, max_slots, steps_per_tick, flags)
        self._ptr = C.c_void_p()
        _check(lib().mmp_server_create(C.byref(cfg), C.byref(self._ptr)), "mmp_server_create")
        self._shape = {}

    def submit(self, prob, params=None) -> int:
        """Queue `prob`; `params` may be its prebuilt prob.to_params() handle."""
        h = params if params is not None else prob.to_params()
        rid = C.c_uint64(0)
        _check(lib().mmp_server_submit(self._ptr, h.ptr(), C.byref(rid)), "mmp_server_submit")
        self._shape[rid.value] = (prob.n_modes, prob.nt)
        return rid.value

    def done(self, rid: int) -> bool:
        d = C.c_int(0)
        _check(lib().mmp_server_poll(self._ptr, rid, C.byref(d)), "mmp_server_poll")
        return bool(d.value)

    def wait(self, rid: int, timeout: float | None = None):
        """(fields complex128 [M][NT], info dict with status, steps and the submit /
        start / done times in seconds since the server started)."""
        M, nt = self._shape[rid]
        out = np.empty((M, nt), dtype=np.complex128)
        info = capi.mmp_request_info()
        rc = lib().mmp_server_wait(self._ptr, rid, -1.0 if timeout is None else float(timeout),
                                   _dptr(out.view(np.float64)), C.byref(info))
        if info.nt != 0:  # info is filled once the request finished; the server then forgets it
            self._shape.pop(rid, None)
        _check(rc, "mmp_server_wait")
        return out, {name: getattr(info, name) for name, _ in info._fields_}

    def close(self):
        if self._ptr:
            lib().mmp_server_destroy(self._ptr)
            self._ptr = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def coupling_from_dense(q: np.ndarray) -> np.ndarray:
    """Dense Q[p, k, l, m] (numpy indexing) to the non-zero list in the order the MEX
    front end inserts it (MATLAB order: p fastest, then k, l, m), as workloads' NZ dtype."""
    from .workloads import NZ_DTYPE
    q = np.asarray(q, dtype=np.float64)
    M = q.shape[0]
    if q.shape != (M, M, M, M):
        raise ValueError("dense coupling must be M x M x M x M")
    flat = np.ascontiguousarray(q.transpose(3, 2, 1, 0)).ravel()   # p fastest in memory
    n = C.c_uint32(0)
    _check(lib().mmp_coupling_from_dense(M, _dptr(flat), None, 0, C.byref(n)), "mmp_coupling_from_dense")
    out = np.zeros(max(n.value, 1), dtype=NZ_DTYPE)   # same layout as mmp_nz
    _check(lib().mmp_coupling_from_dense(M, _dptr(flat), out.ctypes.data_as(C.POINTER(capi.mmp_nz)),
                                         n.value, C.byref(n)), "mmp_coupling_from_dense")
    return out[:n.value]


def write_abs_text(path: str, phi: np.ndarray, phi0: np.ndarray | None = None):
    """The driver's |phi| text dump (mmp_write_abs_text)."""
    a = np.ascontiguousarray(phi, dtype=np.complex128)
    b = None if phi0 is None else np.ascontiguousarray(phi0, dtype=np.complex128)
    M, nt = a.shape
    _check(lib().mmp_write_abs_text(os.fsencode(path), M, nt, None if b is None else _dptr(b.view(np.float64)),
                                    _dptr(a.view(np.float64))), "mmp_write_abs_text")


def write_mat(path: str, Z: float, fields: np.ndarray, cpu_time: float, name: str = "output"):
    """The MEX front end's saved struct {Z, fields, cpu_time} as a Level-5 MAT-file."""
    a = np.ascontiguousarray(fields, dtype=np.complex128)
    M, nt = a.shape
    _check(lib().mmp_write_mat(os.fsencode(path), name.encode(), float(Z), M, nt, _dptr(a.view(np.float64)),
                               float(cpu_time)), "mmp_write_mat")


def dft(x: np.ndarray, inverse: bool = False, fp64: bool = True) -> np.ndarray:
    """Batched transform of the rows of x on the device (Forward_DFT / Inverse_DFT)."""
    a = np.ascontiguousarray(np.atleast_2d(x), dtype=np.complex128)
    out = np.empty_like(a)
    rows, n = a.shape
    _check(lib().mmp_dft(n, rows, 1 if inverse else -1, 1 if fp64 else 0, _dptr(a.view(np.float64)),
                         _dptr(out.view(np.float64))), "mmp_dft")
    return out.reshape(np.shape(x)) if np.ndim(x) == 1 else out
