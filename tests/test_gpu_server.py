"""Served solves (mmp_server_*): every request's fields equal a standalone solve of the
same parameters, whatever else shares its pool, whenever it arrives, and however its
step count falls on the loop's replay boundaries; the memory budget is honoured and
a failing solve fails alone.

Results are compared bit for bit: a served solve runs the same kernels on the same
data as a standalone one (a request joins only a pool whose launch shape, which depends
on its largest solves, is the one it has alone; the pool only adds other solves to the
launch grids)."""
import time

import numpy as np
import pytest

from mm_propagation_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu


def single(mmp, p):
    with mmp.Solver(p) as s:
        s.propagate(p.n_steps)
        return s.result()


def mixed_requests():
    probs = [W.small_case(seed=200 + i, M=1 + i % 4, nt=512, n_steps=5 + 3 * i, nnz_target=6 + 2 * i)
             for i in range(8)]
    probs += [W.small_case(seed=220 + i, M=2, nt=1024, n_steps=7 + i, raman=False) for i in range(3)]
    probs += [W.small_case(seed=230 + i, M=3, nt=512, n_steps=9, order=8) for i in range(2)]
    return [p.replace(flags=capi.MMP_F_FP64) if k % 2 == 0 else p for k, p in enumerate(probs)]


def test_mixed_requests_match_single_solves(mmp):
    probs = mixed_requests()
    with mmp.Server(max_slots=4, steps_per_tick=4) as sv:
        ids = [sv.submit(p) for p in probs]
        outs = [sv.wait(i, timeout=120) for i in ids]
    for k, (p, (out, info)) in enumerate(zip(probs, outs)):
        assert info["status"] == 0, k
        assert info["steps"] == p.n_steps, k
        assert (info["n_modes"], info["nt"]) == (p.n_modes, p.nt)
        assert info["submit_s"] <= info["start_s"] <= info["done_s"], k
        assert np.array_equal(out, single(mmp, p)), k


def test_requests_joining_a_running_pool(mmp):
    # long solves keep the pool busy while short ones arrive, finish and leave
    long = [W.small_case(seed=240 + i, M=3, nt=512, n_steps=120) for i in range(2)]
    short = [W.small_case(seed=250 + i, M=1 + i % 3, nt=512, n_steps=3 + i) for i in range(6)]
    with mmp.Server(max_slots=8, steps_per_tick=2) as sv:
        lid = [sv.submit(p) for p in long]
        time.sleep(0.05)
        sid = []
        for p in short:
            sid.append(sv.submit(p))
            time.sleep(0.01)
        s_out = [sv.wait(i, timeout=120) for i in sid]
        l_out = [sv.wait(i, timeout=120) for i in lid]
    for p, (out, info) in zip(short + long, s_out + l_out):
        assert info["status"] == 0
        assert np.array_equal(out, single(mmp, p))


def test_dense_requests_on_the_tensor_cores_in_a_pool(mmp):
    # dense-Q requests (M >= 6, FP32): the pool's contraction runs on the tensor cores for
    # all of them, as each does alone; they finish at different steps while the pool runs
    probs = []
    for i, (m, n) in enumerate([(6, 7), (7, 4), (6, 10)]):
        p = W.dense15(seed=300 + i, M=m, nt=256, n_steps=n, raman=True)
        probs.append(W.scale_power(p, W.phase_cap_scale(p, per_step=0.05, total=0.3)))
    with mmp.Server(max_slots=4, steps_per_tick=2) as sv:
        ids = [sv.submit(p) for p in probs]
        outs = [sv.wait(i, timeout=120) for i in ids]
    for p, (out, info) in zip(probs, outs):
        assert info["status"] == 0 and info["steps"] == p.n_steps
        with mmp.Solver(p) as s:
            s.propagate(p.n_steps)
            alone, sinfo = s.result(), s.info()
        assert sinfo["tensor_core_contraction"] == 1
        assert np.array_equal(out, alone)


def test_requests_of_different_kernel_shapes_keep_their_own(mmp):
    # With about 200 pair fields per request the contraction runs on the serial-recurrence
    # form (k_contract_sr); a pool chooses its form and tiles from its largest request, so
    # a request that is not tall alone (M + P <= 200: M=20, 177 pair fields) must not be
    # served in a pool of tall ones. Each request here gets the bits of its standalone
    # solve; the tall ones also finish at different steps while their pool runs.
    cases = [(310, 22, 1200, 5, True), (311, 20, 1400, 3, False), (312, 22, 1200, 8, True), (313, 21, 1600, 4, True)]
    probs = [W.small_case(seed=seed, M=m, nt=256, n_steps=n, raman=True, nnz_target=nnz, physical_order=True,
                          peak_w=20.0) for seed, m, nnz, n, _ in cases]
    with mmp.Server(max_slots=4, steps_per_tick=2) as sv:
        ids = [sv.submit(p) for p in probs]
        outs = [sv.wait(i, timeout=120) for i in ids]
    for (seed, _, _, _, tall), p, (out, info) in zip(cases, probs, outs):
        assert info["status"] == 0 and info["steps"] == p.n_steps, seed
        with mmp.Solver(p) as s:
            s.propagate(p.n_steps)
            alone, sinfo = s.result(), s.info()
        assert (sinfo["contract_sub_block"] > 0) == tall, seed
        assert np.array_equal(out, alone), seed


def test_memory_budget_serialises_and_rejects(mmp):
    small = [W.small_case(seed=260 + i, M=2, nt=512, n_steps=6) for i in range(3)]
    with mmp.Server(memory_budget=200 * 1024, steps_per_tick=3) as sv:
        ids = [sv.submit(p) for p in small]
        big = sv.submit(W.small_case(seed=270, M=4, nt=8192, n_steps=2))
        res = [sv.wait(i, timeout=120) for i in ids]
        with pytest.raises(mmp.MMPError) as ei:
            sv.wait(big, timeout=120)
        assert ei.value.code == capi.MMP_ENOMEM
    # one ~100 KB solve at a time: each starts after the previous one finished
    for (_, a), (_, b) in zip(res, res[1:]):
        assert b["start_s"] >= a["done_s"]
    for p, (out, _) in zip(small, res):
        assert np.array_equal(out, single(mmp, p))


def test_failing_request_fails_alone(mmp):
    bad = W.grin2(seed=1, nt=256, n_steps=1000, literal=True)  # diverges (see workloads.grin2)
    good = W.grin2(seed=2, nt=256, n_steps=40, peak_scale=0.01)
    with mmp.Server(steps_per_tick=8) as sv:
        ib = sv.submit(bad)
        ig = sv.submit(good)
        out, info = sv.wait(ig, timeout=120)
        with pytest.raises(mmp.MMPError) as ei:
            sv.wait(ib, timeout=120)
    assert ei.value.code == capi.MMP_ENONFINITE
    assert info["status"] == 0
    assert np.array_equal(out, single(mmp, good))


def test_wait_timeout_keeps_the_request(mmp):
    p = W.small_case(seed=280, M=2, nt=512, n_steps=400)
    with mmp.Server(steps_per_tick=1) as sv:
        rid = sv.submit(p)
        with pytest.raises(mmp.MMPError) as ei:
            sv.wait(rid, timeout=0.0)
        assert ei.value.code == capi.MMP_ETIMEOUT
        out, info = sv.wait(rid, timeout=120)
    assert info["steps"] == 400
    assert np.array_equal(out, single(mmp, p))
