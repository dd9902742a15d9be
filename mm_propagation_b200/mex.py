"""mm_propagation(inputs) — the MATLAB MEX front end of the reference
(matlab/mm_propagation.cpp) over the B200 solver, for callers that drive the solver
with one struct: the same input fields (a dict of numpy arrays / scalars here, indexed
as in MATLAB: dispersion_coefficients[p, j], coupling_coefficients[p, k, l, m],
initial_fields[p, i]), the same structural checks and messages
(checkStructureElements, :341-520), the same n_save chunking and saved files
(:61-101), and the same output struct {Z, fields, cpu_time} (:280-311).

    out = mm_propagation({"n_modes": 2, "fiber_length": 0.1, ..., "savename": "run",
                          "n_save": 4})
    # files run_1.mat, run_2.mat, run_3.mat, run_4.mat; out["fields"] is M x NT complex

Differences from the MEX, on purpose:
* Snapshots carry z across chunks (``z_mode=0``): the MEX calls computeLawsonRK per
  chunk, which restarts z at 0 (src/MultimodePropagation.cpp:158-163), so its
  intermediate results are taken at the wrong z. ``z_mode=1`` reproduces that.
* Numeric checks the MEX does not make (finite values, max|beta2| > 0, ...) come from
  the library (mmp_validate_params) and raise ``InputError`` before any device work.
* ``cpu_time`` is wall time since the call began, like the MEX's omp_get_wtime
  difference; files are written after the last chunk rather than between chunks.
* Bulk arithmetic is FP32 with FP64 phases and field accumulation unless ``fp64=True``.
"""
from __future__ import annotations

import time

import numpy as np

from . import Solver, capi, coupling_from_dense, validate, write_mat
from .workloads import Problem

REQUIRED = ("n_modes", "fiber_length", "dispersion_coefficients", "coupling_coefficients",
            "initial_fields", "time_window", "pulse_width", "n_steps", "method_order",
            "nonlinearity_const")

USAGE = ("Required fields:\n"
         "- n_modes: integer scalar\n"
         "- fiber_length: double scalar\n"
         "- dispersion_coefficients: double array (size: n_modes-by-L)\n"
         "- coupling_coefficients: double array (size: n_modes^4)\n"
         "- initial_fields: double or complex array (size: n_modes-by-N)\n"
         "- time_window: double scalar\n"
         "- pulse_width: double scalar\n"
         "- n_steps: integer scalar\n"
         "- method_order: integer scalar\n"
         "- nonlinearity_const: double scalar\n"
         "Optional fields:\n"
         "- raman_proportion: double scalar\n"
         "- raman_response: double array (size: N)\n"
         "- savename: char array\n"
         "- n_save: integer scalar\n")


class InputError(ValueError):
    """A structural or numeric problem with the input struct; `field` names the field."""

    def __init__(self, msg: str, field: str | None = None):
        super().__init__(msg if field is None else f"Field: {field} is empty. {msg}")
        self.field = field


def _real_array(v) -> bool:
    a = np.asarray(v)
    return a.dtype.kind in "fiu" and a.dtype != np.bool_


def _double_scalar(v) -> bool:
    return _real_array(v) and np.asarray(v).size == 1


def _numeric(v) -> bool:
    a = np.asarray(v)
    return a.dtype.kind in "fiuc" and a.dtype != np.bool_


def check_inputs(s) -> dict:
    """checkArguments + checkStructureElements (matlab/mm_propagation.cpp:326-520).
    Returns the optional-field choices {raman, save, n_save}; raises InputError."""
    if not isinstance(s, dict):
        raise InputError("Input must be a structure.")
    if len(s) < 10:
        raise InputError(USAGE)
    for f in REQUIRED:
        if f not in s:
            raise InputError(f"Field {f} is missing.")
    if not _double_scalar(s["n_modes"]):
        raise InputError("This field must contain an integer scalar.", "n_modes")
    M = int(np.asarray(s["n_modes"]).ravel()[0])
    if not _double_scalar(s["fiber_length"]):
        raise InputError("This field must contain a double scalar.", "fiber_length")
    d = np.asarray(s["dispersion_coefficients"])
    if not _real_array(d) or d.ndim != 2 or d.shape[0] != M:
        raise InputError("This field must contain a n_modes-by-L double array.", "dispersion_coefficients")
    q = np.asarray(s["coupling_coefficients"])
    if q.dtype.kind == "c" or not _numeric(q):
        raise InputError("This field must contain a n_modes^4 double array.", "coupling_coefficients")
    if M > 1 and q.shape != (M, M, M, M):
        raise InputError("This field must contain a n_modes^4 double array.", "coupling_coefficients")
    f0 = np.asarray(s["initial_fields"])
    if not _numeric(f0) or f0.ndim != 2 or f0.shape[0] != M:
        raise InputError("This field must contain a n_modes-by-N double or complex array.", "initial_fields")
    N = f0.shape[1]
    for name, kind in (("time_window", "double"), ("pulse_width", "double"), ("n_steps", "integer"),
                       ("method_order", "integer"), ("nonlinearity_const", "double")):
        if not _double_scalar(s[name]):
            raise InputError(f"This field must contain a{'n' if kind == 'integer' else ''} {kind} scalar.", name)
    raman = save = False
    n_save = 1
    if len(s) > 10:
        raman = "raman_proportion" in s
        if raman:
            if "raman_response" not in s:
                raise InputError("Field raman_response is missing.")
            if not _double_scalar(s["raman_proportion"]):
                raise InputError("This field must contain a double scalar.", "raman_proportion")
            h = np.asarray(s["raman_response"])
            if not _numeric(h) or h.ndim < 1 or h.shape[0] != N:
                raise InputError("This field must contain a N double array.", "raman_response")
        save = "savename" in s
        if save:
            if not isinstance(s["savename"], str):
                raise InputError("This field must contain a char array.", "savename")
            if "n_save" in s:
                if not _double_scalar(s["n_save"]):
                    raise InputError("This field must contain an integer scalar.", "n_save")
                n_save = int(np.asarray(s["n_save"]).ravel()[0])
    return {"raman": raman, "save": save, "n_save": n_save}


def to_problem(s: dict, opts: dict, fp64: bool = False) -> Problem:
    """setInputParameters (matlab/mm_propagation.cpp:108-160) into a Problem."""
    M = int(np.asarray(s["n_modes"]).ravel()[0])
    q = np.asarray(s["coupling_coefficients"], dtype=np.float64).reshape((M, M, M, M))
    f0 = np.asarray(s["initial_fields"]).astype(np.complex128)
    fR = float(np.asarray(s["raman_proportion"]).ravel()[0]) if opts["raman"] else 0.0
    raman_on = opts["raman"] and fR != 0.0   # a zero proportion selects the Raman-off class
    return Problem(
        n_modes=M, nt=f0.shape[1],
        dispersion=np.asarray(s["dispersion_coefficients"], dtype=np.float64),
        coupling=coupling_from_dense(q), initial_fields=f0,
        time_window=float(np.asarray(s["time_window"]).ravel()[0]),
        pulse_width=float(np.asarray(s["pulse_width"]).ravel()[0]),
        fiber_length=float(np.asarray(s["fiber_length"]).ravel()[0]),
        n_steps=int(np.asarray(s["n_steps"]).ravel()[0]),
        method_order=int(np.asarray(s["method_order"]).ravel()[0]),
        nonlinearity_const=float(np.asarray(s["nonlinearity_const"]).ravel()[0]),
        raman_proportion=fR,
        raman_response=(np.real(np.asarray(s["raman_response"])).astype(np.float64).ravel()
                        if raman_on else None),
        raman=raman_on, flags=capi.MMP_F_FP64 if fp64 else 0, name="mex")


def mm_propagation(s: dict, z_mode: int = 0, fp64: bool = False) -> dict:
    """The MEX function (matlab/mm_propagation.cpp:51-101): returns {Z, fields, cpu_time}
    of the last chunk and, with `savename`, writes one MAT-file per chunk."""
    t_start = time.perf_counter()
    opts = check_inputs(s)
    prob = to_problem(s, opts, fp64)
    rc, why = validate(prob)
    if rc != 0:
        raise InputError(why)
    n_save = opts["n_save"]
    if n_save < 1:
        raise InputError("This field must contain an integer scalar.", "n_save")
    with Solver(prob) as sol:
        t_setup = time.perf_counter() - t_start
        fields, Z, elapsed = sol.snapshots(n_save, z_mode)
    cpu = t_setup + elapsed
    if opts["save"]:
        base = s["savename"]
        for i in range(n_save - 1):
            write_mat(f"{base}_{i + 1}.mat", Z[i], fields[i], cpu[i])
        last = base if n_save == 1 else f"{base}_{n_save}"
        write_mat(f"{last}.mat", Z[-1], fields[-1], cpu[-1])
    return {"Z": float(Z[-1]), "fields": fields[-1], "cpu_time": float(cpu[-1])}
