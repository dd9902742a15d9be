"""Parity at the measured configurations' full sizes, a few steps each, against the
oracle (the numpy restatement of the reference's CPU solver, FP64): the 28-mode sweep's
shape at its top member's power and the dense 15-mode shape on the tensor cores.

Tolerances as in test_gpu_parity: relative L2 per mode 1e-5 (FP32 bulk), 1e-11 (FP64).
The reference's per-stage work these cover: src/MultimodePropagation_CPU.cpp:193-229
(pair products, Raman convolution, contraction)."""
import pytest

import mmp_oracle as mo
from mm_propagation_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu


def _run(mmp, prob, steps):
    with mmp.Solver(prob) as s:
        s.propagate(steps)
        return s.result(), s.info()


def test_sweep28_shape_top_member(mmp):
    # M = 28, NT = 65536, order 6, Raman on, ~2000 GRIN non-zeros (313 pair fields), at the
    # sweep's highest power (every member scaled by the one factor the benchmark uses)
    top = W.sweep28(seed=0, index=31)
    prob = W.scale_power(top, W.phase_cap_scale(top))
    steps = 2
    ref = mo.solve(prob, chunks=[steps])
    out32, info = _run(mmp, prob, steps)
    assert info["contract_sub_block"] == 16 and info["raman_recurrence"] == 2, info
    assert info["n_modes"] == 28 and info["nt"] == 65536 and info["n_stages"] == 7
    assert mo.rel_l2_per_mode(out32, ref).max() < 1e-5
    out64, _ = _run(mmp, prob.replace(flags=capi.MMP_F_FP64), steps)
    assert mo.rel_l2_per_mode(out64, ref).max() < 1e-11


def test_dense15_shape_on_tensor_cores(mmp):
    # M = 15, NT = 8192, dense symmetric Q (50625 terms, 120 pair fields), Raman on: the
    # contraction on the tensor cores (TF32 split operands, FP32 sums)
    d = W.dense15(seed=0)
    prob = W.scale_power(d, W.phase_cap_scale(d))
    steps = 2
    ref = mo.solve(prob, chunks=[steps])
    out, info = _run(mmp, prob, steps)
    assert info["tensor_core_contraction"] == 1 and info["n_pair_fields"] == 120, info
    assert mo.rel_l2_per_mode(out, ref).max() < 1e-5
