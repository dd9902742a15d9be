"""Chunked propagation with snapshots (mmp_propagate_snapshots) and the MEX-style
front end on the GPU, against the oracle's restatement of the MEX loop.

Tolerances (relative L2 per mode): FP64 1e-11, FP32 bulk 1e-5, as in the parity tests."""
import numpy as np
import pytest

import mmp_oracle as mo
from mm_propagation_b200 import capi, mex, workloads as W

pytestmark = pytest.mark.gpu

TOL64 = 1e-11
TOL32 = 1e-5


@pytest.mark.parametrize("z_mode", [0, 1])
@pytest.mark.parametrize("n_steps,n_save", [(23, 4), (3, 5), (12, 1)])
def test_snapshots_match_oracle(mmp, z_mode, n_steps, n_save):
    prob = W.small_case(seed=300 + n_steps, M=3, nt=512, n_steps=n_steps).replace(flags=capi.MMP_F_FP64)
    ref, zref = mo.snapshots(prob, n_save, z_mode)
    with mmp.Solver(prob) as s:
        f, z, t = s.snapshots(n_save, z_mode)
    assert np.array_equal(z, zref)
    assert np.all(np.diff(t) >= 0)
    for i in range(n_save):
        assert mo.rel_l2_per_mode(f[i], ref[i]).max() < TOL64, i


def test_continuous_snapshots_end_where_one_call_ends(mmp):
    for flags, tol in ((capi.MMP_F_FP64, 1e-13), (0, 1e-6)):
        prob = W.small_case(seed=310, M=2, nt=1024, n_steps=30).replace(flags=flags)
        with mmp.Solver(prob) as s:
            s.propagate(30)
            one = s.result()
        with mmp.Solver(prob) as s:
            f, _, _ = s.snapshots(7, 0)
        assert mo.rel_l2_per_mode(f[-1], one).max() < tol


def test_snapshots_fp32_within_tolerance(mmp):
    prob = W.small_case(seed=320, M=4, nt=2048, n_steps=40, order=6)
    ref, _ = mo.snapshots(prob, 5, 0)
    with mmp.Solver(prob) as s:
        f, _, _ = s.snapshots(5, 0)
    for i in range(5):
        assert mo.rel_l2_per_mode(f[i], ref[i]).max() < TOL32


def test_mex_front_end_writes_the_chunk_files(mmp, tmp_path):
    sio = pytest.importorskip("scipy.io")
    from test_io import mex_struct
    prob = W.small_case(seed=330, M=2, nt=256, n_steps=10)
    base = str(tmp_path / "run")
    s = mex_struct(prob, savename=base, n_save=3.0)
    out = mex.mm_propagation(s, fp64=True)
    conv = mex.to_problem(s, mex.check_inputs(s), fp64=True)
    ref, zref = mo.snapshots(conv, 3, 0)
    assert out["Z"] == zref[-1]
    assert mo.rel_l2_per_mode(out["fields"], ref[-1]).max() < TOL64
    for i in range(3):
        d = sio.loadmat(f"{base}_{i + 1}.mat", squeeze_me=True, struct_as_record=False)["output"]
        assert d.Z == zref[i]
        assert mo.rel_l2_per_mode(d.fields, ref[i]).max() < TOL64
    assert d.cpu_time == out["cpu_time"] and np.array_equal(d.fields, out["fields"])
