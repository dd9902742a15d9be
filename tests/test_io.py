"""Host-side formats and the MEX-style front end's checks (no kernel launches):
dense coupling input order, the driver's |phi| text dump, the MAT-file struct, and
checkStructureElements' messages."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import mmp_oracle as mo
import mm_propagation_b200 as mmp
from mm_propagation_b200 import mex, workloads as W


def test_coupling_from_dense_matches_mex_order():
    rng = np.random.default_rng(3)
    M = 3
    q = rng.standard_normal((M, M, M, M))
    q[rng.random(q.shape) < 0.6] = 0.0
    got = mmp.coupling_from_dense(q)
    want = mo.coupling_from_dense(q)
    assert len(got) == len(want)
    assert [tuple(int(e[f]) for f in "pklm") + (float(e["value"]),) for e in got] == want


def test_coupling_from_dense_single_mode_and_empty():
    assert len(mmp.coupling_from_dense(np.full((1, 1, 1, 1), 2.5))) == 1
    assert len(mmp.coupling_from_dense(np.zeros((2, 2, 2, 2)))) == 0


def test_write_mat_reads_back_with_scipy(tmp_path):
    sio = pytest.importorskip("scipy.io")
    rng = np.random.default_rng(4)
    phi = rng.standard_normal((3, 64)) + 1j * rng.standard_normal((3, 64))
    path = str(tmp_path / "snap.mat")
    mmp.write_mat(path, 0.125, phi, 3.5)
    d = sio.loadmat(path, squeeze_me=True, struct_as_record=False)
    out = d["output"]
    assert out.Z == 0.125 and out.cpu_time == 3.5
    assert out.fields.shape == (3, 64)
    assert np.array_equal(out.fields, phi)


def test_write_mat_single_sample_and_name(tmp_path):
    sio = pytest.importorskip("scipy.io")
    phi = np.array([[1 + 2j]])
    path = str(tmp_path / "one.mat")
    mmp.write_mat(path, 1.0, phi, 0.0, name="res")
    d = sio.loadmat(path, squeeze_me=False, struct_as_record=True)
    rec = d["res"][0, 0]
    assert rec["fields"].shape == (1, 1) and rec["fields"][0, 0] == 1 + 2j


def test_abs_text_matches_restatement(tmp_path):
    rng = np.random.default_rng(5)
    phi0 = rng.standard_normal((2, 32)) * 1e3 + 1j * rng.standard_normal((2, 32))
    phi = rng.standard_normal((2, 32)) * 1e-4 + 1j * rng.standard_normal((2, 32)) * 1e-6
    path = str(tmp_path / "out.txt")
    mmp.write_abs_text(path, phi, phi0)
    assert open(path).read().splitlines() == mo.abs_text_lines(phi0, phi)


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++ for the iostream check")
def test_abs_text_equals_iostream_formatting(tmp_path):
    # the driver prints with std::ostream defaults; compare against a compiled one-liner
    vals = [0.0, 1.0, 1e-5, 123456.0, 1234567.0, 3.14159265358979, 2.5e-300, 7.0e22, 0.000123456789]
    src = tmp_path / "p.cpp"
    src.write_text("#include <iostream>\n#include <complex>\nint main(){double v;\n"
                   "while(std::cin>>v) std::cout<<std::abs(std::complex<double>(v,0.))<<std::endl;}\n")
    exe = str(tmp_path / "p")
    subprocess.run(["g++", "-O0", "-o", exe, str(src)], check=True)
    r = subprocess.run([exe], input="\n".join(repr(v) for v in vals), capture_output=True, text=True,
                       check=True)
    phi = np.array([vals], dtype=np.complex128)
    path = str(tmp_path / "o.txt")
    mmp.write_abs_text(path, phi)
    assert open(path).read().splitlines() == r.stdout.splitlines()


def mex_struct(prob, **extra):
    M = prob.n_modes
    q = np.zeros((M, M, M, M))
    for e in prob.coupling:
        q[e["p"], e["k"], e["l"], e["m"]] = e["value"]
    s = {"n_modes": float(M), "fiber_length": prob.fiber_length,
         "dispersion_coefficients": prob.dispersion, "coupling_coefficients": q,
         "initial_fields": prob.initial_fields, "time_window": prob.time_window,
         "pulse_width": prob.pulse_width, "n_steps": float(prob.n_steps),
         "method_order": float(prob.method_order), "nonlinearity_const": prob.nonlinearity_const}
    if prob.raman:
        s["raman_proportion"] = prob.raman_proportion
        s["raman_response"] = prob.raman_response
    s.update(extra)
    return s


@pytest.mark.parametrize("mutate,msg", [
    (lambda s: [s.pop(k) for k in ("pulse_width", "raman_proportion", "raman_response")],
     "Required fields"),
    (lambda s: s.update(x=1) or s.pop("n_steps"), "Field n_steps is missing."),
    (lambda s: s.update(n_modes=np.array([2.0, 2.0])), "n_modes"),
    (lambda s: s.update(dispersion_coefficients=np.zeros((3, 3))), "n_modes-by-L"),
    (lambda s: s.update(coupling_coefficients=np.zeros((2, 2, 2))), "n_modes^4"),
    (lambda s: s.update(coupling_coefficients=np.zeros((2, 2, 2, 2), complex)), "n_modes^4"),
    (lambda s: s.update(initial_fields=np.zeros((3, 16))), "n_modes-by-N"),
    (lambda s: s.update(method_order=np.array([4.0, 6.0])), "method_order"),
    (lambda s: s.pop("raman_response"), "Field raman_response is missing."),
    (lambda s: s.update(raman_response=np.zeros(7)), "N double array"),
    (lambda s: s.update(savename=3), "char array"),
])
def test_mex_structure_checks(mutate, msg):
    s = mex_struct(W.small_case(seed=1, M=2, nt=64))
    mutate(s)
    with pytest.raises(mex.InputError) as ei:
        mex.check_inputs(s)
    assert msg in str(ei.value)


def test_mex_optional_fields():
    s = mex_struct(W.small_case(seed=1, M=2, nt=64, raman=False))
    assert mex.check_inputs(s) == {"raman": False, "save": False, "n_save": 1}
    s["n_save"] = 4.0  # without savename the MEX ignores n_save
    s["x1"] = 0
    assert mex.check_inputs(s)["n_save"] == 1
    s["savename"] = "run"
    assert mex.check_inputs(s) == {"raman": False, "save": True, "n_save": 4}


def test_mex_to_problem_follows_setinputparameters():
    prob = W.small_case(seed=2, M=3, nt=128)
    s = mex_struct(prob)
    p = mex.to_problem(s, mex.check_inputs(s))
    assert p.n_modes == 3 and p.nt == 128 and p.raman
    assert [tuple(int(e[f]) for f in "pklm") for e in p.coupling] == \
        [e[:4] for e in mo.coupling_from_dense(s["coupling_coefficients"])]
    assert np.array_equal(p.initial_fields, prob.initial_fields)
    s["raman_proportion"] = 0.0   # a zero proportion selects the Raman-off class
    assert not mex.to_problem(s, mex.check_inputs(s)).raman
