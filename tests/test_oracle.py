"""CPU checks of the oracle: the FFTW-API shim against numpy.fft, the numpy
restatement against the reference's own compiled solver (golden fixtures and
live runs), and the tableau data. No GPU involved."""
import numpy as np
import pytest

import mmp_oracle as mo
import ref_lib
from fixtures import load, names
from mm_propagation_b200 import workloads as W

needs_ref = pytest.mark.skipif(not ref_lib.available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("n", [1, 2, 8, 64, 1000, 4096, 16384])
def test_fftw_shim_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert np.abs(ref_lib.fft(x, -1) - np.fft.fft(x)).max() <= 1e-13 * max(1, np.abs(x).sum())
    assert np.abs(ref_lib.fft(x, +1) - np.fft.ifft(x) * n).max() <= 1e-13 * max(1, np.abs(x).sum())


@pytest.mark.parametrize("name", names())
def test_restatement_matches_golden(name):
    prob, chunks, ref = load(name)
    out = mo.solve(prob, chunks)
    err = mo.rel_l2_per_mode(out, ref).max()
    assert err < 1e-12, f"{name}: relL2 {err:.3e}"


@needs_ref
@pytest.mark.parametrize("seed,M,nt,order,raman", [(31, 2, 128, 4, True), (32, 3, 256, 6, False),
                                                   (33, 4, 64, 8, True)])
def test_restatement_matches_reference_live(seed, M, nt, order, raman):
    prob = W.small_case(seed=seed, M=M, nt=nt, n_steps=6, order=order, raman=raman)
    ref, _ = ref_lib.run(prob)
    assert mo.rel_l2_per_mode(mo.solve(prob), ref).max() < 1e-12


@needs_ref
def test_reference_z_snapshots_match_reference_chunked_calls():
    # the MEX loop with z_mode 1: snapshot i is the reference after i+1 computeLawsonRK calls
    prob = W.small_case(seed=34, M=3, nt=128, n_steps=11)
    snaps, Z = mo.snapshots(prob, 3, z_mode=1)
    chunks = [3, 3, 5]
    for i in range(3):
        ref, _ = ref_lib.run(prob, chunks[:i + 1])
        assert mo.rel_l2_per_mode(snaps[i], ref).max() < 1e-12
    assert np.allclose(Z, np.cumsum(chunks) * prob.fiber_length / prob.n_steps, rtol=1e-15)


def test_continuous_snapshots_end_at_the_single_call_result():
    prob = W.small_case(seed=35, M=3, nt=128, n_steps=23)
    snaps, _ = mo.snapshots(prob, 4, z_mode=0)
    assert mo.rel_l2_per_mode(snaps[-1], mo.solve(prob)).max() < 1e-13


def test_pair_quirk_is_active_for_lexicographic_grin2():
    s = mo.OracleSolver(W.grin2(nt=64, n_steps=10))
    assert s.unique_pairs == [0, 2, 1, 3]


@pytest.mark.parametrize("tab", [mo.butcher4(), mo.butcher7(1.0), mo.butcher11()])
def test_tableau_consistency(tab):
    a, b, c = tab
    s = len(b)
    assert len(a) == s
    for i in range(s):
        assert abs(sum(a[i]) - c[i]) < 1e-14
    assert abs(sum(b) - 1.0) < 1e-14
    assert abs(sum(bi * ci for bi, ci in zip(b, c)) - 0.5) < 1e-14      # order >= 2
    assert abs(sum(bi * ci * ci for bi, ci in zip(b, c)) - 1 / 3) < 1e-14  # order >= 3


def test_butcher7_lambda_mu_weights_do_not_sum_to_one():
    # src/RungeKutta.cpp:107-113: sum b = 1/120 + 27/20 - 8/15 + 11/120 = 11/12 for every lambda
    for lam in (1.0, 2.0, -3.0):
        _, b, _ = mo.butcher7_lambda_mu(lam, 0.5)
        assert abs(sum(b) - 11 / 12) < 1e-14
