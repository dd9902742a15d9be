"""The byte and flop models behind the bench line's roofline fractions (bench.stage_bytes,
bench.stage_flops), checked against the per-sample sums written out by hand for the
6-mode RK4 batch and the 28-mode order-6 sweep."""
import bench
from mm_propagation_b200 import workloads as W


def _pairs(prob):
    c = prob.coupling
    return len({(min(int(l), int(m)), max(int(l), int(m)))
                for l, m, v in zip(c["l"], c["m"], c["value"]) if v != 0})


def test_k_nu_bytes_rk4():
    # FP32 (8-byte complex), RK4: three intermediate stages read sigma and write N_i and U
    # (3 x 8), read psi_hat's FP32 copy (8), no stored N_j (a[i+1][j] = 0 for j < i); the
    # last stage also reads and writes psi_hat in FP64 (2 x 16), writes its copy (8) and
    # reads N_0..N_2 (3 x 8): (32 + 32 + 32 + 88) / 4 = 46 bytes per mode-sample
    prob = W.grin6(seed=0)
    a, b, c, s = bench.batch_tableau(4)
    per = bench.stage_bytes(prob, s, a, b, 8, _pairs(prob), 2)
    M, NT = prob.n_modes, prob.nt
    assert per["nu"] == 46 * M * NT
    assert per["pair"] == M * NT * 8            # the tile aggregates read U
    assert per["contract"] == 2 * M * NT * 8    # read U, write sigma


def test_contract_flops_sweep():
    # NT (8 nnz (1 + r) + 6 P) for the Kerr and Raman terms and the pair products, plus
    # 24 P NT when the recurrence runs inside the contraction tiles
    prob = W.sweep28(seed=0, index=31)
    P = _pairs(prob)
    nnz = int((prob.coupling["value"] != 0).sum())
    f = bench.stage_flops(prob, P, nnz, 2, recurrence_in_contract=True)
    NT = prob.nt
    assert f["contract"] == NT * (16.0 * nnz + 6.0 * P) + 24.0 * P * NT
    assert f["pair"] == 24.0 * P * NT
