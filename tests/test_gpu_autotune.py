"""The autotuner (csrc/solver.cu, autotune): every launch parameter it may pick gives
results within tolerance of the oracle; its choice is reported in mmp_info and cached per
shape; the steps it times leave no trace in the solves it tuned.

Parameters: the transform kernels' row split (cluster_ctas: the minimal CTA set or twice
as many), the contraction tile (contract_tile) and the graph branches (graph_branches).
Tolerance: relative L2 per mode 1e-5 (FP32 bulk), as in test_gpu_parity."""
import numpy as np
import pytest

import mmp_oracle as mo
from mm_propagation_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL32 = 1e-5


def _tall(seed, M=22, nnz=1200, nt=256):
    # about 200 pair fields: the serial-recurrence contraction (k_contract_sr)
    return W.small_case(seed=seed, M=M, nt=nt, n_steps=3, raman=True, nnz_target=nnz, physical_order=True,
                        peak_w=20.0)


def _batch_run(mmp, probs, steps):
    with mmp.Batch(probs) as b:
        b.propagate(steps)
        return [b.result(i) for i in range(len(probs))], b.info(0)


@pytest.mark.parametrize("kind", ["serial_recurrence", "term_loop"])
def test_every_tile_and_branch_candidate_matches_oracle(mmp, monkeypatch, kind):
    if kind == "serial_recurrence":
        probs = [_tall(140), _tall(141, M=20, nnz=1400)]
    else:  # k_contract with the recurrence in its tiles
        probs = [W.small_case(seed=142 + i, M=3, nt=1024, n_steps=4) for i in range(2)]
    refs = [mo.solve(p) for p in probs]
    for tile in (64, 128, 256):
        for groups in (1, 2):
            monkeypatch.setenv("MMP_CONTRACT_TILE", str(tile))
            monkeypatch.setenv("MMP_GROUPS", str(groups))
            outs, info = _batch_run(mmp, probs, probs[0].n_steps)
            assert (info["contract_tile"], info["graph_branches"]) == (tile, groups), info
            assert (info["contract_sub_block"] > 0) == (kind == "serial_recurrence")
            for out, ref in zip(outs, refs):
                assert mo.rel_l2_per_mode(out, ref).max() < TOL32, (tile, groups)


@pytest.mark.parametrize("nt", [16384, 65536])
def test_every_row_split_candidate_matches_oracle(mmp, monkeypatch, nt):
    prob = W.small_case(seed=150, M=2, nt=nt, n_steps=3, window=40.0, nnz_target=8)
    ref = mo.solve(prob)
    ctas = []
    for xc in (0, 1):
        monkeypatch.setenv("MMP_ROW_SPLIT", str(xc))
        with mmp.Solver(prob) as s:
            s.propagate(prob.n_steps)
            out, info = s.result(), s.info()
        ctas.append(info["cluster_ctas"])
        assert mo.rel_l2_per_mode(out, ref).max() < TOL32, xc
    assert ctas[1] == 2 * ctas[0]


@pytest.mark.parametrize("fp64,nt", [(False, 4096), (False, 8192), (False, 32768), (True, 2048), (True, 4096),
                                     (True, 8192), (True, 16384)])
def test_every_split_row_geometry_matches_oracle(mmp, monkeypatch, fp64, nt):
    # the row-split variants not covered above: rows dealt out to 2, 4 or 8 CTAs in runs
    # of 32 bytes (4 FP32 or 2 FP64 samples), combined by one radix-(C G) butterfly
    from mm_propagation_b200 import capi
    prob = W.small_case(seed=151, M=2, nt=nt, n_steps=3, window=40.0 if nt >= 16384 else 10.0, nnz_target=8)
    ref = mo.solve(prob)
    prob = prob.replace(flags=prob.flags | (capi.MMP_F_FP64 if fp64 else 0))
    ctas = []
    for xc in (0, 1):
        monkeypatch.setenv("MMP_ROW_SPLIT", str(xc))
        with mmp.Solver(prob) as s:
            s.propagate(prob.n_steps)
            out, info = s.result(), s.info()
        ctas.append(info["cluster_ctas"])
        assert mo.rel_l2_per_mode(out, ref).max() < (1e-11 if fp64 else TOL32), xc
    assert ctas[1] == 2 * ctas[0]


def test_tuned_choice_is_reported_cached_and_leaves_no_trace(mmp, monkeypatch):
    probs = [_tall(160 + i) for i in range(4)]
    outs, info = _batch_run(mmp, probs, 3)  # tuned here (or taken from the cache)
    assert info["autotuned"] == 1
    choice = (info["cluster_ctas"], info["contract_tile"], info["graph_branches"])
    outs2, info2 = _batch_run(mmp, probs, 3)  # the cached choice for the same shape
    assert info2["autotuned"] == 1
    assert (info2["cluster_ctas"], info2["contract_tile"], info2["graph_branches"]) == choice
    # the same parameters fixed by hand (nothing timed): the tuned batch's timing steps
    # were undone exactly, so the results are bitwise the same
    monkeypatch.setenv("MMP_ROW_SPLIT", "1" if choice[0] > 1 else "0")
    monkeypatch.setenv("MMP_CONTRACT_TILE", str(choice[1]))
    monkeypatch.setenv("MMP_GROUPS", str(choice[2]))
    outs3, info3 = _batch_run(mmp, probs, 3)
    assert info3["autotuned"] == 0
    for a, b, c in zip(outs, outs2, outs3):
        assert np.array_equal(a, c) and np.array_equal(b, c)
