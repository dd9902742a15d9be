"""GPU solver parity: libmmp_b200 through the C ABI against the reference's own
CPU solver (golden fixtures) and the numpy restatement (live, small sizes).

Tolerances (relative L2 per mode, ||phi_p - ref_p|| / ||ref_p||):
  FP64 path (MMP_F_FP64):  1e-11  — same algorithm in FP64; differences are
                                    rounding and transform order only.
  FP32-bulk path:          1e-5   — FP32 transforms/contraction, FP64 phase and
                                    field accumulation.
"""
import numpy as np
import pytest

import mmp_oracle as mo
from fixtures import load, names
from mm_propagation_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu

TOL64 = 1e-11
TOL32 = 1e-5


@pytest.fixture
def pinned(monkeypatch):
    """The launch parameters the autotuner picks for batches (row split, contraction tile,
    graph branches), fixed to the defaults single solves use: batch members and single
    solves then run the same kernels and give the same bits."""
    monkeypatch.setenv("MMP_ROW_SPLIT", "0")
    monkeypatch.setenv("MMP_CONTRACT_TILE", "256")
    monkeypatch.setenv("MMP_GROUPS", "1")


def run(mmp, prob, chunks, flags=0):
    prob = prob.replace(flags=prob.flags | flags)
    with mmp.Solver(prob) as s:
        for c in chunks:
            s.propagate(c)
        return s.result(), s.info()


@pytest.mark.parametrize("name", names())
@pytest.mark.parametrize("fp64", [True, False])
def test_golden(mmp, name, fp64):
    prob, chunks, ref = load(name)
    out, _ = run(mmp, prob, chunks, capi.MMP_F_FP64 if fp64 else 0)
    err = mo.rel_l2_per_mode(out, ref).max()
    assert err < (TOL64 if fp64 else TOL32), f"{name} fp64={fp64}: relL2 {err:.3e}"


def test_quirk_reported(mmp):
    prob, chunks, _ = load("grin2_quirk_raman")
    _, info = run(mmp, prob, chunks)
    assert info["pair_quirk_active"] == 1 and info["n_pairs"] == 4
    prob2, chunks2, _ = load("m3_physical_order")
    _, info2 = run(mmp, prob2, chunks2)
    assert info2["pair_quirk_active"] == 0


@pytest.mark.parametrize("order", [4, 6, 8])
@pytest.mark.parametrize("raman", [True, False])
def test_orders_live(mmp, order, raman):
    prob = W.small_case(seed=40 + order, M=3, nt=256, n_steps=8, order=order, raman=raman)
    ref = mo.solve(prob)
    for fp64, tol in ((True, TOL64), (False, TOL32)):
        out, _ = run(mmp, prob, [prob.n_steps], capi.MMP_F_FP64 if fp64 else 0)
        assert mo.rel_l2_per_mode(out, ref).max() < tol


def test_physical_pairs_flag(mmp):
    prob = W.small_case(seed=51, M=3, nt=256, n_steps=10)
    ref = mo.solve(prob, physical_pairs=True)
    out, info = run(mmp, prob, [10], capi.MMP_F_FP64 | capi.MMP_F_PHYSICAL_PAIRS)
    assert mo.rel_l2_per_mode(out, ref).max() < TOL64
    assert info["pair_quirk_active"] == 0
    # and the default reproduces the reference's slot indexing, which differs here
    quirk = mo.solve(prob)
    assert mo.rel_l2_per_mode(quirk, ref).max() > 1e-6


def test_butcher7_lambda_mu(mmp):
    prob = W.small_case(seed=52, M=2, nt=128, n_steps=6).replace(
        rk_variant=capi.MMP_RK_BUTCHER7_LAMBDA_MU, rk_lambda=2.0, rk_mu=0.5)
    ref = mo.solve(prob)
    out, info = run(mmp, prob, [6], capi.MMP_F_FP64)
    assert info["n_stages"] == 7
    assert mo.rel_l2_per_mode(out, ref).max() < TOL64


def test_continuous_chunks_equal_one_call(mmp):
    # with MMP_F_CONTINUOUS, computeLawsonRK(5) + (7) is the same propagation as (12)
    prob = W.small_case(seed=53, M=3, nt=256, n_steps=12)
    one, _ = run(mmp, prob, [12], capi.MMP_F_FP64)
    two, info = run(mmp, prob, [5, 7], capi.MMP_F_FP64 | capi.MMP_F_CONTINUOUS)
    assert mo.rel_l2_per_mode(two, one).max() < 1e-13
    assert abs(info["z"] - 12 * info["delta_z"]) < 1e-15
    # without it, the reference's z reset makes them differ
    reset, _ = run(mmp, prob, [5, 7], capi.MMP_F_FP64)
    assert mo.rel_l2_per_mode(reset, one).max() > 1e-8


def test_batch_members_match_single_solves(mmp, pinned):
    probs = [W.small_case(seed=60 + i, M=m, nt=512, n_steps=10, nnz_target=8 + 4 * i)
             for i, m in enumerate([2, 3, 1, 4])]
    probs = [p.replace(flags=capi.MMP_F_FP64) for p in probs]
    singles = [run(mmp, p, [10])[0] for p in probs]
    with mmp.Batch(probs) as b:
        b.propagate(10)
        for i, p in enumerate(probs):
            assert np.array_equal(b.result(i), singles[i]), i


def test_set_fields_restarts(mmp):
    prob = W.small_case(seed=70, M=2, nt=256, n_steps=10).replace(flags=capi.MMP_F_FP64)
    other = W.small_case(seed=71, M=2, nt=256, n_steps=10)
    with mmp.Solver(prob) as s:
        s.propagate(10)
        s.set_fields(other.initial_fields)
        s.propagate(10)
        out = s.result()
    ref = mo.solve(prob.replace(initial_fields=other.initial_fields))
    assert mo.rel_l2_per_mode(out, ref).max() < TOL64


def test_noarg_propagate_uses_floor(mmp):
    prob, chunks, ref = load("m2_noarg")
    out, info = run(mmp, prob, chunks, capi.MMP_F_FP64)
    assert mo.rel_l2_per_mode(out, ref).max() < TOL64
    assert info["steps_done"] == int(np.floor(info["z_final"] / info["delta_z"]))


def test_energy_monitor_conserved_without_raman(mmp):
    prob = W.grin2(seed=3, nt=1024, n_steps=1000, peak_scale=0.01, raman=False)
    with mmp.Solver(prob.replace(flags=capi.MMP_F_FP64)) as s:
        s.propagate(200)
        e, _ = s.monitors()
    assert len(e) == 200
    e0 = (np.abs(prob.initial_fields) ** 2).sum() * prob.time_window / prob.nt
    assert abs(e[0] / e0 - 1) < 1e-6
    assert np.abs(e / e[0] - 1).max() < 1e-6


def test_set_fields_rejects_nonfinite_and_keeps_the_solve(mmp):
    # set_fields checks the fields on the device copy, before any of the solve's state changes
    prob = W.small_case(seed=90, M=3, nt=1024, n_steps=4)
    ref = mo.solve(prob)
    bad = prob.initial_fields.copy()
    bad[1, 17] = np.inf
    with mmp.Solver(prob) as s:
        for v in (np.nan, np.inf):
            bad[1, 17] = v
            with pytest.raises(mmp.MMPError) as ei:
                s.set_fields(bad)
            assert ei.value.code == capi.MMP_EINVAL
            assert "not finite" in mmp.lib().mmp_last_error().decode()
        s.propagate(prob.n_steps)
        out = s.result()
    assert mo.rel_l2_per_mode(out, ref).max() < TOL32


def test_nonfinite_is_reported(mmp):
    # the literal reading of the four-entry pattern diverges (see workloads.grin2)
    prob = W.grin2(seed=1, nt=256, n_steps=1000, literal=True)
    with mmp.Solver(prob) as s:
        with pytest.raises(mmp.MMPError) as ei:
            s.propagate(400)
    assert ei.value.code == capi.MMP_ENONFINITE


@pytest.mark.parametrize("nt", [32768, 65536])
@pytest.mark.parametrize("fp64", [True, False])
def test_cluster_rows_live(mmp, nt, fp64):
    # rows that span a thread-block cluster (FP32 from 2^15, FP64 from 2^14 samples)
    prob = W.small_case(seed=80, M=2, nt=nt, n_steps=3, window=40.0, nnz_target=8)
    ref = mo.solve(prob)
    out, info = run(mmp, prob, [3], capi.MMP_F_FP64 if fp64 else 0)
    assert info["cluster_ctas"] >= 2
    assert mo.rel_l2_per_mode(out, ref).max() < (TOL64 if fp64 else TOL32)


def test_grin6_full_rows_live(mmp):
    # full-size rows of the 6-mode workload (M=6, NT=16384, 60 GRIN non-zeros,
    # Raman on), 8 steps, at a power where RK4 is stable (at 5 kW the reference's
    # own solver already loses energy within 20 steps of this step size)
    prob = W.grin6(seed=1, n_steps=5000, peak_total_w=500.0)
    ref = mo.solve(prob, [8])
    a, _ = run(mmp, prob, [8])
    b, _ = run(mmp, prob, [8], capi.MMP_F_FP64)
    assert mo.rel_l2_per_mode(b, ref).max() < TOL64
    assert mo.rel_l2_per_mode(a, ref).max() < TOL32


def two_term_response(nt, window):
    """A Raman response that is not one damped sinusoid (two of them): the solver must
    take the FFT convolution for it."""
    dt = window / nt
    t = np.arange(nt) * dt
    h = np.exp(-t / 0.032) * np.sin(t / 0.0122) + 0.3 * np.exp(-t / 0.1) * np.sin(t / 0.05)
    return h / (h.sum() * dt)


@pytest.mark.parametrize("fp64", [True, False])
def test_raman_fft_path_for_a_general_response(mmp, fp64):
    prob = W.small_case(seed=90, M=3, nt=1024, n_steps=8)
    prob = prob.replace(raman_response=two_term_response(1024, prob.time_window))
    ref = mo.solve(prob)
    out, info = run(mmp, prob, [8], capi.MMP_F_FP64 if fp64 else 0)
    assert info["raman_recurrence"] == 0
    assert mo.rel_l2_per_mode(out, ref).max() < (TOL64 if fp64 else TOL32)


@pytest.mark.parametrize("fp64", [True, False])
@pytest.mark.parametrize("nt,window", [(256, 10.0), (4096, 10.0), (65536, 40.0)])
def test_raman_recurrence_matches_fft_convolution(mmp, monkeypatch, fp64, nt, window):
    # h_R of the reference driver's form: the recurrence path, checked against the FFT
    # path on the same solve and against the oracle
    prob = W.small_case(seed=91, M=3, nt=nt, n_steps=6, window=window, nnz_target=10)
    fl = capi.MMP_F_FP64 if fp64 else 0
    out_r, info_r = run(mmp, prob, [6], fl)            # inside the contraction tiles
    monkeypatch.setenv("MMP_RAMAN_FUSED", "0")
    out_s, info_s = run(mmp, prob, [6], fl)            # row scan
    monkeypatch.setenv("MMP_RAMAN_FFT", "1")
    out_f, info_f = run(mmp, prob, [6], fl)            # FFT convolution
    assert (info_r["raman_recurrence"], info_s["raman_recurrence"], info_f["raman_recurrence"]) == (2, 1, 0)
    tol = 1e-12 if fp64 else 2e-6
    assert mo.rel_l2_per_mode(out_r, out_f).max() < tol
    assert mo.rel_l2_per_mode(out_s, out_f).max() < tol
    ref = mo.solve(prob)
    assert mo.rel_l2_per_mode(out_r, ref).max() < (TOL64 if fp64 else TOL32)


@pytest.mark.parametrize("fp64", [True, False])
@pytest.mark.parametrize("raman", [True, False])
def test_dense_contraction_matches_term_loop_and_oracle(mmp, monkeypatch, fp64, raman):
    # fully symmetric dense Q (the dense 15-mode workload's construction at M = 5)
    prob = W.dense15(seed=92, M=5, nt=512, n_steps=8, raman=raman)
    prob = W.scale_power(prob, W.phase_cap_scale(prob, per_step=0.05, total=0.4))
    fl = capi.MMP_F_FP64 if fp64 else 0
    out_d, info_d = run(mmp, prob, [8], fl)
    monkeypatch.setenv("MMP_DENSE", "0")
    out_s, info_s = run(mmp, prob, [8], fl)
    assert (info_d["dense_contraction"], info_s["dense_contraction"]) == (1, 0)
    assert mo.rel_l2_per_mode(out_d, out_s).max() < (1e-12 if fp64 else 2e-6)
    assert mo.rel_l2_per_mode(out_d, mo.solve(prob)).max() < (TOL64 if fp64 else TOL32)


def test_dense_contraction_forced_on_a_sparse_quirky_case(mmp, monkeypatch):
    # GRIN-pattern coupling with the reference's pair-slot mapping active: the dense form
    # built from the resolved terms must reproduce it
    prob = W.small_case(seed=93, M=4, nt=256, n_steps=6, nnz_target=20).replace(flags=capi.MMP_F_FP64)
    monkeypatch.setenv("MMP_DENSE", "1")
    out, info = run(mmp, prob, [6])
    assert info["dense_contraction"] == 1 and info["pair_quirk_active"] == 1
    assert mo.rel_l2_per_mode(out, mo.solve(prob)).max() < TOL64


def test_fp32_monitors_match_fp64(mmp):
    # energy and photon-number monitors (center frequency of 1550 nm light) of the FP32-bulk
    # path against the FP64 path: FP64 accumulation in both, FP32 photon weights in the former
    prob = W.grin2(seed=4, nt=1024, n_steps=1000, peak_scale=0.01).replace(center_frequency=1215.2)
    mons = []
    for fl in (0, capi.MMP_F_FP64):
        with mmp.Solver(prob.replace(flags=fl)) as s:
            s.propagate(100)
            mons.append(s.monitors())
    (e32, p32), (e64, p64) = mons
    assert len(e32) == len(p32) == 100 and p64.min() > 0
    assert np.abs(e32 / e64 - 1).max() < 1e-6
    assert np.abs(p32 / p64 - 1).max() < 1e-5


def _dense_case(seed, M, nt, n_steps, raman):
    prob = W.dense15(seed=seed, M=M, nt=nt, n_steps=n_steps, raman=raman)
    return W.scale_power(prob, W.phase_cap_scale(prob, per_step=0.05, total=0.3))


@pytest.mark.parametrize("raman", [True, False])
def test_dense_contraction_on_tensor_cores(mmp, monkeypatch, raman):
    # fully symmetric Q at M = 8 (36 pair fields: two full K chunks of 16 and a partial
    # one): the tensor-core form (TF32 operands split hi + lo, FP32 sums) against the
    # register-blocked FP32 form and the oracle
    prob = _dense_case(94, 8, 1024, 6, raman)
    out_t, info_t = run(mmp, prob, [6])
    monkeypatch.setenv("MMP_TC", "0")
    out_s, info_s = run(mmp, prob, [6])
    assert (info_t["tensor_core_contraction"], info_s["tensor_core_contraction"]) == (1, 0)
    assert info_t["dense_contraction"] == info_s["dense_contraction"] == 1
    assert mo.rel_l2_per_mode(out_t, out_s).max() < 2e-6
    assert mo.rel_l2_per_mode(out_t, mo.solve(prob)).max() < TOL32


def test_dense_contraction_on_tensor_cores_15_modes(mmp, monkeypatch):
    # the dense 15-mode workload's shape: 120 pair fields in 8 K chunks, N = 240 columns
    prob = _dense_case(95, 15, 1024, 4, True)
    out_t, info_t = run(mmp, prob, [4])
    monkeypatch.setenv("MMP_TC", "0")
    out_s, _ = run(mmp, prob, [4])
    assert info_t["tensor_core_contraction"] == 1
    assert mo.rel_l2_per_mode(out_t, out_s).max() < 2e-6


def test_tensor_core_batch_members_match_single_solves(mmp, pinned):
    # solves of different M in one batch: each tile's MMA shape comes from its own solve
    probs = [_dense_case(96 + i, m, 512, 5, True) for i, m in enumerate([6, 8, 7])]
    singles = [run(mmp, p, [5])[0] for p in probs]
    with mmp.Batch(probs) as b:
        b.propagate(5)
        assert b.info(0)["tensor_core_contraction"] == 1
        for i in range(len(probs)):
            assert np.array_equal(b.result(i), singles[i]), i


def test_raman_recurrence_in_tall_tiles(mmp, monkeypatch):
    # over 200 pair fields (328 with the reference's pair-slot mapping): U and all pair
    # fields do not fit in a 64-sample tile. Three routes: the serial recurrence per pair
    # field in 16-sample sub-blocks (k_contract_sr, the default), the pair fields held in
    # chunks with the warp-scan recurrence (k_contract_pc) and the row scan (Raman rows
    # through HBM); against each other and the oracle
    prob = W.small_case(seed=97, M=26, nt=512, n_steps=3, nnz_target=1800)
    ref = mo.solve(prob)
    for fl, tol in ((0, 2e-6), (capi.MMP_F_FP64, 1e-12)):
        out_r, info_r = run(mmp, prob, [3], fl)
        monkeypatch.setenv("MMP_CONTRACT_SR", "0")
        out_t, info_t = run(mmp, prob, [3], fl)
        monkeypatch.setenv("MMP_PAIR_CHUNK", "0")
        out_s, info_s = run(mmp, prob, [3], fl)
        monkeypatch.delenv("MMP_PAIR_CHUNK")
        monkeypatch.delenv("MMP_CONTRACT_SR")
        assert (info_r["raman_recurrence"], info_t["raman_recurrence"], info_s["raman_recurrence"]) == (2, 2, 1)
        assert info_r["n_pair_fields"] > 200
        assert info_r["contract_sub_block"] == 16 and info_r["contract_pair_chunk"] == 0
        assert 0 < info_t["contract_pair_chunk"] < info_t["n_pair_fields"] and info_t["contract_sub_block"] == 0
        assert info_s["contract_pair_chunk"] == 0 and info_s["contract_sub_block"] == 0
        assert mo.rel_l2_per_mode(out_r, out_t).max() < tol
        assert mo.rel_l2_per_mode(out_t, out_s).max() < tol
        for out in (out_r, out_t):
            assert mo.rel_l2_per_mode(out, ref).max() < (TOL64 if fl else TOL32)


def _tall_case(seed, raman, M=22, nnz=1200, nt=256, n_steps=3):
    # physical pair order (no pair-slot quirk), about 200 pair fields: a tall tile
    return W.small_case(seed=seed, M=M, nt=nt, n_steps=n_steps, raman=raman, nnz_target=nnz,
                        physical_order=True, peak_w=20.0)


@pytest.mark.parametrize("raman", [True, False])
@pytest.mark.parametrize("order", [4, 6])
def test_serial_recurrence_contraction_against_oracle(mmp, monkeypatch, raman, order):
    # k_contract_sr: Raman on (recurrence from the tile carries) and off (W = V), FP32 with
    # the packed two-lane FMA and FP64; against the oracle and the term loop it replaces
    prob = _tall_case(120 + order, raman).replace(method_order=order)
    ref = mo.solve(prob)
    for fl, tol in ((0, TOL32), (capi.MMP_F_FP64, TOL64)):
        out, info = run(mmp, prob, [prob.n_steps], fl)
        assert info["contract_sub_block"] == 16 and info["contract_tile"] == 256, info
        assert info["n_pair_fields"] > 150
        assert mo.rel_l2_per_mode(out, ref).max() < tol
        monkeypatch.setenv("MMP_CONTRACT_SR", "0")
        out_o, info_o = run(mmp, prob, [prob.n_steps], fl)
        monkeypatch.delenv("MMP_CONTRACT_SR")
        assert info_o["contract_sub_block"] == 0
        assert mo.rel_l2_per_mode(out, out_o).max() < (2e-6 if fl == 0 else 1e-12)


@pytest.mark.parametrize("seed,M,nnz", [(170, 36, 1500), (172, 40, 1000)])
def test_serial_recurrence_beyond_32_modes(mmp, seed, M, nnz):
    # more than 32 modes: two rounds of the phase-B plan and two staged U items per thread
    # (M * 8 sample pairs > 256 threads); 313 / 241 pair fields
    prob = _tall_case(seed, True, M=M, nnz=nnz)
    ref = mo.solve(prob)
    for fl, tol in ((0, TOL32), (capi.MMP_F_FP64, TOL64)):
        out, info = run(mmp, prob, [prob.n_steps], fl)
        assert info["contract_sub_block"] == 16 and info["n_modes"] == M, info
        assert mo.rel_l2_per_mode(out, ref).max() < tol


def test_serial_recurrence_batch_members_match_single_solves(mmp, pinned):
    # members of different M and coupling in one batch, each a tall tile on its own too
    # (so its single solve runs the same kernel): each CTA reads its own solve's merged
    # terms, pairs and mode order
    probs = [_tall_case(130, True), _tall_case(131, True, M=24, nnz=1500), _tall_case(134, True, M=23, nnz=1300)]
    singles = [run(mmp, p, [3])[0] for p in probs]
    with mmp.Batch(probs) as b:
        b.propagate(3)
        assert b.info(0)["contract_sub_block"] == 16
        for i in range(len(probs)):
            assert np.array_equal(b.result(i), singles[i]), i


def test_dense_contraction_on_tensor_cores_16_modes(mmp, monkeypatch):
    # the largest tensor-core shape: N = 256 accumulator columns per part (all of TMEM),
    # 136 pair fields in 9 K chunks (the last one partial)
    prob = _dense_case(98, 16, 256, 3, True)
    out_t, info_t = run(mmp, prob, [3])
    monkeypatch.setenv("MMP_TC", "0")
    out_s, _ = run(mmp, prob, [3])
    assert info_t["tensor_core_contraction"] == 1 and info_t["n_pair_fields"] == 136
    assert mo.rel_l2_per_mode(out_t, out_s).max() < 2e-6
