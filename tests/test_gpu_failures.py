"""Failure detection on the device, without faulting it.

The reference checks no return code at all (src/MultimodePropagation_GPU.cu:43-44);
this library turns each failure into a status the host reads:
  * a device-side bounded wait that runs out -> MMP_ETIMEOUT (the contraction kernels'
    first wait for their tile copy is given 0 polls through MMP_TILE_WAIT_POLLS, so it
    gives up at once; the copy still lands before the CTA leaves, and the context stays
    usable, which the next solve on the same device shows);
  * a device allocation that fails -> MMP_ENOMEM, with nothing leaked (injected by
    mmp_debug_fail_alloc; live allocations counted by mmp_debug_live_allocations);
  * the FP64 energy monitor leaving its band -> MMP_EDRIFT.
"""
import numpy as np
import pytest

import mmp_oracle
from mm_propagation_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu


def _solve(mmp, prob, steps):
    with mmp.Solver(prob) as s:
        s.propagate(steps)
        return s.result(), s.info()


def _expect(mmp, code, fn):
    with pytest.raises(mmp.MMPError) as ei:
        fn()
    assert ei.value.code == code, str(ei.value)
    return str(ei.value)


# the three contraction kernels that wait for a tile copy: term loop (k_contract),
# tensor cores (k_contract_tc, dense Q at 6 modes), pair-chunked tall tiles (k_contract_pc)
def _cases():
    small = W.small_case(seed=11, M=3, nt=512, n_steps=6, raman=True)
    dense = W.dense15(seed=6, M=6, nt=256, n_steps=4, raman=True)
    dense = W.scale_power(dense, W.phase_cap_scale(dense, per_step=0.05, total=0.2))
    # about 200 pair fields: a tall tile; the pair-chunked kernel is forced (the default for
    # tall tiles, k_contract_sr, makes no asynchronous copies and has no wait to run out)
    tall = W.small_case(seed=12, M=22, nt=256, n_steps=3, raman=True, nnz_target=1200, physical_order=True,
                        peak_w=20.0)
    return [("k_contract", small, {}, lambda i: i["tensor_core_contraction"] == 0 and i["contract_pair_chunk"] == 0),
            ("k_contract_tc", dense, {}, lambda i: i["tensor_core_contraction"] == 1),
            ("k_contract_pc", tall, {"MMP_CONTRACT_SR": "0"}, lambda i: i["contract_pair_chunk"] > 0)]


@pytest.mark.parametrize("kernel,prob,env,check", _cases(), ids=lambda x: x if isinstance(x, str) else "")
def test_bounded_tile_wait_runs_out_and_reports_timeout(mmp, monkeypatch, kernel, prob, env, check):
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    monkeypatch.setenv("MMP_TILE_WAIT_POLLS", "0")
    s = mmp.Solver(prob)
    monkeypatch.delenv("MMP_TILE_WAIT_POLLS")
    with s:
        assert check(s.info()), (kernel, s.info())
        msg = _expect(mmp, capi.MMP_ETIMEOUT, lambda: s.propagate(prob.n_steps))
        assert "bounded wait" in msg
    # the device is still usable: the same solve with the default bound matches the oracle
    out, info = _solve(mmp, prob, prob.n_steps)
    assert check(info)
    err = float(mmp_oracle.rel_l2_per_mode(out, mmp_oracle.solve(prob)).max())
    assert err < 1e-5, (kernel, err)


def test_allocation_failure_reports_enomem_and_leaks_nothing(mmp):
    lib = capi.load()
    prob = W.small_case(seed=13, M=2, nt=256, n_steps=4, raman=True)
    ref, _ = _solve(mmp, prob, 4)  # device set-up (twiddle tables) happens here, once
    live0 = lib.mmp_debug_live_allocations()
    failed = []
    try:
        # allocation 0: the batch's descriptors, 1: the solve's state block, 2: the
        # monitor buffers (first propagate); from 3 on the solve runs through
        for after in range(4):
            lib.mmp_debug_fail_alloc(after)
            try:
                out, _ = _solve(mmp, prob, 4)
                assert np.array_equal(out, ref)
            except mmp.MMPError as e:
                assert e.code == capi.MMP_ENOMEM, str(e)
                failed.append(after)
            lib.mmp_debug_fail_alloc(-1)
            assert lib.mmp_debug_live_allocations() == live0, after
    finally:
        lib.mmp_debug_fail_alloc(-1)
    assert failed == [0, 1, 2]


def test_server_admission_failure_reports_enomem_and_recovers(mmp):
    lib = capi.load()
    prob = W.small_case(seed=14, M=3, nt=512, n_steps=8, raman=True)
    ref, _ = _solve(mmp, prob, prob.n_steps)
    live0 = lib.mmp_debug_live_allocations()
    sv = mmp.Server()
    try:
        lib.mmp_debug_fail_alloc(0)  # the pool's first allocation, on the worker thread
        rid = sv.submit(prob)
        msg = _expect(mmp, capi.MMP_ENOMEM, lambda: sv.wait(rid, timeout=120))
        assert "out of memory" in msg, msg  # the worker's error text reaches this thread
        lib.mmp_debug_fail_alloc(-1)
        out, info = sv.wait(sv.submit(prob), timeout=120)
        assert info["status"] == 0
        assert np.array_equal(out, ref)  # served == standalone, after the failure
    finally:
        lib.mmp_debug_fail_alloc(-1)
        sv.close()
    assert lib.mmp_debug_live_allocations() == live0


def test_energy_drift_limit(mmp):
    # Raman off: the 2-mode coupling conserves energy (the FP64 monitor stays within 1e-6
    # over these steps, as the monitor test in test_gpu_parity checks)
    prob = W.grin2(seed=3, nt=1024, n_steps=1000, peak_scale=0.01, raman=False)
    with mmp.Solver(prob.replace(flags=capi.MMP_F_FP64)) as s:
        s.set_energy_drift_limit(1e-6)
        s.propagate(100)
        e, _ = s.monitors()
        assert np.abs(e / e[0] - 1).max() < 1e-6
    with mmp.Solver(prob) as s:
        s.set_energy_drift_limit(1e-15)  # below FP32 bulk rounding: must trip
        msg = _expect(mmp, capi.MMP_EDRIFT, lambda: s.propagate(100))
        assert "energy" in msg
        s.set_fields(prob.initial_fields)  # clears the status and the reference energy
        s.set_energy_drift_limit(0.0)
        s.propagate(100)
    with mmp.Solver(prob.replace(flags=capi.MMP_F_NO_MONITORS)) as s:
        _expect(mmp, capi.MMP_ESTATE, lambda: s.set_energy_drift_limit(1e-3))
