#!/usr/bin/env python
"""bench.py — throughput of the Lawson–RK step (mode-samples·steps/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    torchrun --nproc-per-node N bench.py --gpus N ...     (replicas, one per GPU)

Workload (default "sweep28", the large batched sweep, the largest configuration that
fits one GPU): M=28, NT=65536, 20 ps window, 2 m, 10000 steps per solve, RK order 6,
Raman on, ~2000 GRIN-symmetric non-zeros; a batch of 32 independent solves whose total
peak powers are log-spaced over the batch, advanced by the same launches. One bench
step is R Lawson–RK steps of the whole batch. value = all ranks' B*M*NT*R*K / device
time (CUDA events on the solver's stream, max over ranks).

--workload grin6 | grin2 | dense15 measures the other configurations the same way
(see WORKLOADS and make_problem); --workload serve the mixed request stream.

Accuracy (rank 0, N=1): the timed batch itself runs with z carried across calls, so
its warm-up, profiling and timed calls compose into one solve; after the timed region
it is advanced to the workload's accuracy step count (1000 steps, or the full solve)
and every member's result is compared, per mode, with the same batch run in FP64.

The peak power is set where the reference's own FP64 solver is stable and
converged at this step size (see workloads.grin6 and the accuracy block); the
throughput per step does not depend on it.

--impl reference runs the reference's own CPU solver (oracle/_ref/libmmref.so,
built from its unmodified sources) on the host cores: one process per batch
member, K RK steps each, all cores busy.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mode-samples·steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed bench steps (each R RK steps)")
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=tuple(WORKLOADS) + ("serve",), default="sweep28",
                    help="sweep28: the large batched sweep (default); grin6, grin2, dense15: the "
                         "other configurations; serve: the mixed request stream")
    ap.add_argument("--batch", type=int, default=None, help="independent solves per GPU")
    ap.add_argument("--rk-per-step", type=int, default=None, help="RK steps per bench step")
    ap.add_argument("--order", type=int, default=4, help="RK order (grin6)")
    ap.add_argument("--peak-w", type=float, default=None, help="grin6: total peak power per solve (W, default 8)")
    ap.add_argument("--fp64", action="store_true", help="all-FP64 arithmetic")
    ap.add_argument("--e2e-iters", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=None, help="RK steps of an e2e solve (default per workload)")
    ap.add_argument("--cpu-steps", type=int, default=None, help="RK steps per process in the CPU sample")
    ap.add_argument("--acc-steps", type=int, default=None, help="RK steps of the FP32-vs-FP64 check")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--profile-only", action="store_true", help="short run for ncu captures")
    ap.add_argument("--requests", type=int, default=512, help="serve: requests in the stream")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: mean Poisson arrival rate (1/s)")
    ap.add_argument("--sub-rate", type=float, default=None,
                    help="serve: also run the stream at this arrival rate (default: 0.7 of the capacity "
                         "measured at --rate); 0 skips it")
    ap.add_argument("--check", type=int, default=4, help="serve: requests re-solved in FP64 for relL2")
    args = ap.parse_args()
    w = WORKLOADS.get(args.workload, WORKLOADS["grin6"])
    if args.steps is None:
        args.steps = w.get("steps", 40)
    if args.warmup is None:
        args.warmup = w.get("warmup", 5)
    if args.batch is None:
        args.batch = w["batch"]
    if args.rk_per_step is None:
        args.rk_per_step = w["rk"]
    if args.e2e_steps is None:
        args.e2e_steps = w["e2e"]
    if args.cpu_steps is None:
        args.cpu_steps = w["cpu"]
    if args.acc_steps is None:
        args.acc_steps = w["acc"]
    return args


# ---- process-group plumbing ----------------------------------------------------------------
class Dist:
    """One process per GPU (torchrun env). The ranks are replicas: each runs its own batch
    of independent solves; the only collectives are a barrier and the max of the timings.
    Backend NCCL on GPUs; MMP_DIST_BACKEND=gloo runs the same plumbing on CPU (tests)."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = os.environ.get("MMP_DIST_BACKEND", "nccl")
        self.pg = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as td
            if self.backend == "nccl":
                torch.cuda.set_device(self.local)
            td.init_process_group(self.backend, timeout=datetime.timedelta(seconds=300))
            self.pg = td

    def _device(self):
        return "cuda" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self.pg:
            import torch
            t = torch.zeros(1, device=self._device())
            self.pg.all_reduce(t)
            if self.backend == "nccl":
                torch.cuda.synchronize()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self._device())
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---- clocks during the timed region --------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None
        self.idx = gpu_index

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---- workload ------------------------------------------------------------------------------
# Per workload: batch per GPU, RK steps per bench step, default timed / warm-up bench
# steps, RK steps of an e2e solve (None: the full n_steps), RK steps of the CPU sample,
# RK steps of the FP32-vs-FP64 check on the timed batch (None: the full solve).
WORKLOADS = {
    "sweep28": dict(batch=32, rk=20, steps=30, warmup=3, e2e=100, cpu=1, acc=1000,
                    desc="sweep28: M=28, NT=65536, 20 ps, 2 m, 10000 steps, order 6, ~2000 GRIN terms, Raman on, "
                         "peaks log-spaced over the batch"),
    "grin6": dict(batch=32, rk=50, steps=40, warmup=5, e2e=None, cpu=6, acc=None,
                  desc="grin6: M=6, NT=16384, 20 ps, 1 m, 5000 steps, GRIN Q, Raman on"),
    # 40 RK steps per bench step: warm-up and timed steps together make the 1000-step solve,
    # so the accuracy check compares full solves (beyond the fibre FP64 itself stops
    # converging at this step size)
    "grin2": dict(batch=128, rk=40, steps=20, warmup=5, e2e=None, cpu=20, acc=None,
                  desc="grin2: M=2, NT=4096, 10 ps, 0.1 m, 1000 steps, the four-entry pattern, Raman on"),
    "dense15": dict(batch=16, rk=10, steps=40, warmup=5, e2e=400, cpu=2, acc=1000,
                    desc="dense15: M=15, NT=8192, 20 ps, 0.5 m, 4000 steps, dense symmetric Q (50625 terms), Raman on"),
}


def make_problem(workload: str, seed: int, order: int, peak_w, flags: int = 0):
    """One member of a workload (module level: the CPU worker processes build theirs
    the same way). Power levels: grin6 at `peak_w` total (default 8 W: at 10 W the worst of
    the 32 seeded members' FP32-bulk errors over the full solve was 1.15e-5, at 8 W
    4.0e-6); grin2 at 1/100 of the stated 10 kW / 1 kW; dense15 and sweep28 at the stated
    powers lowered by one factor (for sweep28 the top of the ladder's) until the nonlinear
    phase is at most 5.6e-3 rad per step and 28 rad per fiber (the 6-mode workload's
    levels at 10 W): at the stated powers RK4/RK6 at these step lengths diverge."""
    from mm_propagation_b200 import workloads as W
    if workload == "grin6":
        return W.grin6(seed=seed, order=order, peak_total_w=8.0 if peak_w is None else peak_w, flags=flags)
    if workload == "grin2":
        return W.grin2(seed=seed, peak_scale=0.01, flags=flags)
    if workload == "dense15":
        p = W.dense15(seed=seed, flags=flags)
        return W.scale_power(p, W.phase_cap_scale(p))
    if workload == "sweep28":
        return W.scale_power(W.sweep28(seed=0, index=seed % 32, flags=flags), _sweep28_scale())
    raise ValueError(workload)


_SWEEP_SCALE = []


def _sweep28_scale():
    """One power factor for the whole sweep: the top member's phase cap (cached)."""
    from mm_propagation_b200 import workloads as W
    if not _SWEEP_SCALE:
        _SWEEP_SCALE.append(W.phase_cap_scale(W.sweep28(seed=0, index=31)))
    return _SWEEP_SCALE[0]


def make_batch_problems(args, rank: int, fp64=None):
    """The batch's members. z is carried across propagate calls (MMP_F_CONTINUOUS), so
    every call on the batch continues one solve of each member."""
    from mm_propagation_b200 import capi
    fp64 = args.fp64 if fp64 is None else fp64
    flags = (capi.MMP_F_FP64 if fp64 else 0) | capi.MMP_F_CONTINUOUS
    return [make_problem(args.workload, 1000 * rank + i, args.order, args.peak_w, flags)
            for i in range(args.batch)]


def stage_bytes(prob, tab_s, a, b, bt, pairs, raman_path):
    """Algorithmic DRAM bytes per launch for each kernel kind, one solve, averaged
    over the stages of a step (complex elements of bt bytes; psi_hat is FP64).
    raman_path (mmp_info.raman_recurrence): 0 pair fields by FFT convolution (k_pair),
    1 by the row recurrence (k_raman_scan), 2 by the recurrence inside the contraction
    tiles (k_raman_agg + k_raman_carry; their per-tile carries, under 1% of the bytes,
    are not counted)."""
    M, NT = prob.n_modes, prob.nt
    P = pairs if prob.raman else 0
    if raman_path == 0:
        pair = (M + P + 1) * NT * bt                   # read U, write R, read H_R
    elif raman_path == 1:
        pair = (M + P) * NT * bt                       # read U, write R
    else:
        pair = M * NT * bt                             # read U
    contract = (2 * M + (P if raman_path in (0, 1) else 0)) * NT * bt  # read U (and R), write sigma
    nu = 0.0
    for i in range(tab_s):
        last = i == tab_s - 1
        rows = 3 * M * bt                              # read sigma, write N_i, write U
        if last:
            # read and write psi_hat (FP64), write its copy in T (FP32 solves), read the N_j
            rows += 2 * M * 16 + (M * bt if bt == 8 else 0)
            rows += sum(1 for j in range(tab_s) if b[j] != 0 and j != i) * M * bt
        else:
            # read psi_hat's copy in T (psi_hat itself in FP64), read the stored N_j
            rows += M * bt + sum(1 for j in range(i) if a[i + 1][j] != 0) * M * bt  # N_i is in registers
        nu += rows * NT
    return {"pair": pair, "contract": contract, "nu": nu / tab_s}


def stage_flops(prob, pairs, n_terms, raman_path, recurrence_in_contract=False):
    """Algorithmic FP32 flops per launch for each kernel kind, one solve, on the
    per-sample model of the hot path: 5 N log2 N per complex transform; the Raman
    recurrence 24 flops per sample and pair field (pair product, two complex first-order
    steps, output); the contraction 6 per pair field (pair products) plus 8 per non-zero
    term for the Kerr part and 8 more for the Raman part (NT (6 P + 8 nnz (1 + r)));
    about 70 per sample for k_nu's phase factors and stage combination. When the
    contraction kernel runs the recurrence through its own tiles (k_contract, k_contract_sr)
    the recurrence's flops are its own; the pair kernel then only forms the tile
    aggregates (the same 24 per sample and pair field)."""
    M, NT = prob.n_modes, prob.nt
    P = pairs if prob.raman else 0
    r = 1 if prob.raman else 0
    fft = 5.0 * NT * math.log2(NT)
    if raman_path == 0:
        pair = P * (2 * fft + 12 * NT)
    else:
        pair = P * NT * 24.0
    contract = NT * (8.0 * n_terms * (1 + r) + 6.0 * pairs)
    if recurrence_in_contract:
        contract += P * NT * 24.0
    nu = M * (2 * fft + 70.0 * NT)
    return {"pair": pair, "contract": contract, "nu": nu}


def tc_mma_flops(prob, pairs):
    """TF32 work the tensor-core contraction issues per solve and launch: per tile of 128
    samples and chunk of 16 pair fields, 2 products (Re, Im) x 3 split terms (hi hi, hi lo,
    lo hi) of 128 x 16 M x 16 MMA work, i.e. 2 * 3 * 2 * 16 ceil(P/16) * 16 M flops per sample."""
    chunks = -(-pairs // 16)
    return 2 * 3 * 2.0 * 16 * chunks * 16 * prob.n_modes * prob.nt


def tf32_peak_tflops():
    """Dense TF32 tensor peak: the measured BF16 burst (MEASURED_PEAKS.json bf16_tflops)
    halved, TF32 MMAs running at half the BF16 rate on this part (nominal 1.1 vs 2.25
    PFLOP/s); 1.1 PFLOP/s nominal when no measurement is present."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        if d.get("bf16_tflops"):
            return float(d["bf16_tflops"]) / 2, "measured BF16 burst (MEASURED_PEAKS.json bf16_tflops) / 2"
    return 1100.0, "nominal dense TF32"


def ncu_tf32_peak_tflops():
    """The TF32 tensor peak ncu reports for this part
    (sm__ops_path_tensor_op_utchmma_src_tf32_dst_fp32_sparsity_off ... peak_sustained_elapsed,
    in ops/ns) in the committed k_contract_tc summary; None when absent."""
    p = os.path.join(ROOT, "profiles", "k_contract_tc_dense15.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if "peak_sustained_elapsed.per_second" in line and "tf32" in line:
            cells = [c.strip() for c in line.split("|")]
            try:
                return float(cells[2].replace(",", "")) * 1e9 / 1e12
            except (ValueError, IndexError):
                return None
    return None


def fp32_peak_tflops():
    """Nominal FP32 (non-tensor) peak: 148 SMs x 128 lanes x 2 flops x max SM clock.
    MEASURED_PEAKS.json carries no FP32 figure."""
    mhz = 1965.0
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            mhz = float(json.load(f).get("sm_max_mhz", mhz))
    return 148 * 128 * 2 * mhz * 1e6 / 1e12


def read_measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_ncu_traffic(kind: str, workload: str):
    """dram bytes per launch from the committed ncu summary, scaled to this batch."""
    p = os.path.join(ROOT, "profiles", f"{kind}_{workload}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_solve_per_launch:"):
            return float(line.split(":")[1])
    return None


# ---- CPU side: the reference's own solver in worker processes ------------------------------
def _ref_worker(q, spec):
    os.environ["OMP_NUM_THREADS"] = str(spec["threads"])
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np  # noqa: F401
    import ref_lib
    prob = make_problem(spec["workload"], spec["seed"], spec["order"], spec["peak_w"])
    out, sec = ref_lib.run(prob, [spec["steps"]])
    q.put((spec["index"], sec, out if spec["keep"] else None, ref_lib.threads(prob.n_modes)))


def run_reference_cpu(workload: str, n_members: int, steps: int, order: int, peak_w, keep=None):
    """The reference's CPU solver on min(n_members, cores) batch members at once, one
    process each, `steps` RK steps; members are taken from the top of the batch down
    (for the sweep: the highest powers). Returns timings and member `keep`'s output."""
    ncpu = os.cpu_count() or 1
    nproc = max(1, min(n_members, ncpu))
    threads = max(1, ncpu // nproc)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = []
    members = [n_members - 1 - i for i in range(nproc)]
    for m in members:
        spec = {"workload": workload, "seed": m, "order": order, "peak_w": peak_w, "steps": steps, "threads": threads,
                "index": m, "keep": keep == m}
        p = ctx.Process(target=_ref_worker, args=(q, spec))
        p.start()
        procs.append(p)
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    secs = [r[1] for r in res]
    kept = next((r[2] for r in res if r[0] == keep), None)
    eff_threads = res[0][3][1]
    return {"procs": nproc, "threads_per_proc": threads, "effective_omp_threads": eff_threads,
            "max_seconds": max(secs), "kept_output": kept, "members": members}


def reference_arm(args, dist):
    if dist.rank != 0:
        return None
    probe = make_problem(args.workload, 0, args.order, args.peak_w)
    steps = max(1, min(args.steps, {"grin6": 20, "grin2": 20, "dense15": 2}.get(args.workload, 1)))
    r = run_reference_cpu(args.workload, args.batch, steps, args.order, args.peak_w)
    work = r["procs"] * probe.n_modes * probe.nt * steps
    value = work / r["max_seconds"]
    cores = r["procs"] * r["effective_omp_threads"]
    sample = (f"{r['procs']} concurrent reference solves (one process each, batch members), "
              f"{steps} RK steps each, OMP threads/process {r['threads_per_proc']} "
              f"(reference uses {r['effective_omp_threads']})")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": args.gpus, "steps": steps, "warmup": 0,
        "ms_per_step": 1000.0 * r["max_seconds"] / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, probe, dist.world),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def workload_config(args, probe, world):
    nnz = int((probe.coupling["value"] != 0).sum())
    cfg = {"workload": f"{WORKLOADS[args.workload]['desc']}; M={probe.n_modes}, NT={probe.nt}, "
                       f"RK order {probe.method_order}, {nnz} non-zero Q entries; batch of {args.batch} "
                       f"independent solves per GPU",
           "global_batch": args.batch * world, "rk_steps_per_bench_step": args.rk_per_step,
           "peak_total_w": probe.notes.get("peak_total_w"), "power_scale": probe.notes.get("power_scale", 1.0),
           "precision": "fp64" if args.fp64 else "fp32-bulk+fp64-phase/accum",
           "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (batch state > 126 MB)"}
    if args.workload == "sweep28":
        top = make_problem(args.workload, args.batch - 1, args.order, args.peak_w)
        cfg["peak_total_w"] = [probe.notes.get("peak_total_w"), top.notes.get("peak_total_w")]
        cfg["peaks"] = "log-spaced over the batch (first, last member)"
    return cfg


def rel_l2_modes(x, y):
    """Relative L2 error of x against y, per mode (rows)."""
    import numpy as np
    return np.sqrt((np.abs(x - y) ** 2).sum(-1) / (np.abs(y) ** 2).sum(-1))


# ---- our arm -------------------------------------------------------------------------------
def ours_arm(args, dist):
    import numpy as np
    import mm_propagation_b200 as mmp
    from mm_propagation_b200 import capi

    lib = mmp.lib()
    probs = make_batch_problems(args, dist.rank)
    probe = probs[0]
    M, NT = probe.n_modes, probe.nt
    R, K = args.rk_per_step, args.steps
    batch = mmp.Batch(probs)
    info = batch.info(0)
    n_pairs = info["n_pair_fields"]
    state_mb = sum((p.n_modes * p.nt * 16 * 2 + (p.n_stages + 2) * p.n_modes * p.nt * (16 if args.fp64 else 8)
                    + n_pairs * p.nt * (16 if args.fp64 else 8)) for p in probs) / 1e6
    steps_run = 0  # RK steps the batch has advanced (z carried: one solve per member)
    for _ in range(args.warmup):
        batch.propagate(R)
        steps_run += R
    info = batch.info(0)  # after the first propagate: the autotuned kernel choices
    chosen = {"row_ctas": info["cluster_ctas"], "raman_recurrence": info["raman_recurrence"],
              "dense_contraction": info["dense_contraction"], "graph_branches": info["graph_branches"],
              "tensor_core_contraction": info["tensor_core_contraction"],
              "contract_pair_chunk": info["contract_pair_chunk"], "contract_sub_block": info["contract_sub_block"],
              "contract_tile": info["contract_tile"], "autotuned": info["autotuned"]}
    if args.profile_only:
        print(json.dumps({"kernels_chosen": chosen}))
        batch.propagate(R)
        batch.result(0)  # getResult (k_result) once
        return None
    # per-kernel device times (un-graphed, one event pair per launch)
    prof = batch.profile(2)
    steps_run += 2
    # timed region
    clocks = Clocks(dist.local)
    dist.barrier()
    clocks.start()
    time.sleep(0.3)
    l0 = lib.mmp_kernel_launch_count()
    ms = batch.propagate_timed(R, K)
    launches = lib.mmp_kernel_launch_count() - l0
    clk = clocks.stop()
    steps_run += R * K
    dist.barrier()
    ms_max = dist.max(ms)
    work = dist.world * args.batch * M * NT * R * K
    value = work / (ms_max / 1000.0)

    # accuracy of the timed batch itself (rank 0, N=1): advanced to the check's step count,
    # every member against the same batch in FP64
    acc = None
    if dist.rank == 0 and dist.world == 1 and not args.no_accuracy and not args.fp64:
        target = probe.n_steps if args.acc_steps is None else min(args.acc_steps, probe.n_steps)
        if target > steps_run:
            batch.propagate(target - steps_run)
            steps_run = target
        out32 = [batch.result(i) for i in range(len(probs))]
        probs64 = make_batch_problems(args, dist.rank, fp64=True)
        with mmp.Batch(probs64) as b64:
            b64.propagate(steps_run)
            out64 = [b64.result(i) for i in range(len(probs64))]
        per_mode = [rel_l2_modes(a, b) for a, b in zip(out32, out64)]
        top = int(np.argmax([p.notes.get("peak_total_w", 0.0) for p in probs]))
        acc = {"rk_steps": steps_run, "of_n_steps": probe.n_steps, "tolerance": 1e-5,
               "relL2_max_fp32_vs_fp64": float(max(e.max() for e in per_mode)),
               "relL2_fp32_vs_fp64_per_member": [float(e.max()) for e in per_mode],
               "top_member": top, "top_member_peak_total_w": probs[top].notes.get("peak_total_w"),
               "relL2_fp32_vs_fp64_top_member_per_mode": [float(x) for x in per_mode[top]],
               "source": "the timed FP32 batch (warm-up, profiling and timed calls with z carried, then "
                         "advanced to rk_steps) vs the same members run in FP64 for rk_steps"}
        # convergence of FP64 itself at this z: the top member at twice the steps
        p2 = probs64[top].replace(n_steps=2 * probe.n_steps)
        with mmp.Solver(p2) as s2:
            s2.propagate(2 * steps_run)
            acc["relL2_max_fp64_vs_fp64_2x_steps_top_member"] = float(rel_l2_modes(out64[top], s2.result()).max())
        del out32, out64

    # e2e through the public API with pinned host buffers
    import torch
    pin_in = [torch.from_numpy(np.ascontiguousarray(p.initial_fields)).pin_memory() for p in probs]
    pin_out = [torch.empty((p.n_modes, p.nt), dtype=torch.complex128).pin_memory() for p in probs]
    nsteps = probe.n_steps if args.e2e_steps is None else min(args.e2e_steps, probe.n_steps)
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_iters):
        for i in range(len(probs)):
            batch.set_fields(i, pin_in[i].numpy())
        batch.propagate(nsteps)
        for i in range(len(probs)):
            batch.result(i, pin_out[i].numpy())
    t_e2e = dist.max(time.perf_counter() - t0)
    e2e_value = dist.world * args.batch * M * NT * nsteps * args.e2e_iters / t_e2e
    h2d = sum(p.n_modes * p.nt * 16 for p in probs)

    # roofline of the dominant kernel
    bt = 16 if args.fp64 else 8
    tab = batch_tableau(probe.method_order)
    raman_path = info["raman_recurrence"]
    n_terms = int((probe.coupling["value"] != 0).sum())
    per = stage_bytes(probe, tab[3], tab[0], tab[1], bt, n_pairs, raman_path)
    tc = bool(info.get("tensor_core_contraction", 0))
    pc = bool(info.get("contract_pair_chunk", 0))
    sr = bool(info.get("contract_sub_block", 0))
    flops = stage_flops(probe, n_pairs, n_terms, raman_path, recurrence_in_contract=(raman_path == 2))
    names = {"pair": ("k_pair", "k_raman_scan", "k_raman_agg+k_raman_carry")[raman_path],
             "contract": ("k_contract_tc" if tc else "k_contract_sr" if sr else "k_contract_pc" if pc
                          else "k_contract"), "nu": "k_nu"}
    share = {k: prof[k]["ms_per_launch"] * prof[k]["launches"] for k in prof}
    tot = sum(share.values())
    dom = max(share, key=share.get)
    peak, peak_kind = read_measured_peaks()
    fpeak = fp32_peak_tflops()
    kernels = {}
    for k in prof:
        if not prof[k]["launches"]:
            continue
        t = prof[k]["ms_per_launch"] / 1e3
        bytes_launch = per[k] * args.batch
        flops_launch = flops[k] * args.batch
        ach = bytes_launch / t / 1e9
        t_hbm, t_fp32 = bytes_launch / (peak * 1e9), flops_launch / (fpeak * 1e12)
        kernels[k] = {"name": names[k], "ms_per_launch": prof[k]["ms_per_launch"], "share": share[k] / tot,
                      "alg_bytes_per_launch": bytes_launch, "achieved_gbs": ach, "frac": ach / peak,
                      "alg_flops_per_launch": flops_launch, "achieved_tflops": flops_launch / t / 1e12,
                      "fp32_frac": flops_launch / t / 1e12 / fpeak,
                      "roofline_bound": "hbm" if t_hbm >= t_fp32 else "fp32",
                      "roofline_frac": max(t_hbm, t_fp32) / t}
    tpeak, tpeak_src = tf32_peak_tflops()
    if tc and "contract" in kernels:
        # the dense contraction on the tensor cores: its issued TF32 MMA work (3 split products)
        # and the useful GEMM work (8 M^4 NT per stage and solve) against the TF32 peak
        kc = kernels["contract"]
        tflops = tc_mma_flops(probe, n_pairs) * args.batch
        useful = 8.0 * probe.n_modes ** 4 * probe.nt * args.batch
        t = kc["ms_per_launch"] / 1e3
        t_tensor = tflops / (tpeak * 1e12)
        npeak = ncu_tf32_peak_tflops()
        kc.update({"tensor_flops_per_launch": tflops, "achieved_tensor_tflops": tflops / t / 1e12,
                   "tensor_frac": tflops / t / 1e12 / tpeak,
                   "ncu_tf32_peak_tflops": npeak,
                   "tensor_frac_of_ncu_tf32_peak": (tflops / t / 1e12 / npeak) if npeak else None,
                   "useful_gemm_flops_per_launch": useful, "useful_gemm_tflops": useful / t / 1e12,
                   "useful_gemm_frac_of_measured_bf16_burst": useful / t / 1e12 / (2 * tpeak),
                   "roofline_bound": "tensor" if t_tensor >= kc["alg_bytes_per_launch"] / (peak * 1e9) else "hbm",
                   "roofline_frac": max(t_tensor, kc["alg_bytes_per_launch"] / (peak * 1e9)) / t})
    traffic_solve = read_ncu_traffic(names[dom].split("+")[0], args.workload)
    kd = kernels[dom]
    if tc and dom == "contract":
        roof = {"bound": "tensor", "kernel": names[dom], "achieved": kd["achieved_tensor_tflops"], "peak": tpeak,
                "unit": "TFLOP/s", "frac": kd["tensor_frac"], "peak_source": tpeak_src,
                "tensor_flops_per_launch": kd["tensor_flops_per_launch"],
                "note": "achieved counts the issued TF32 MMA work (3 split products per product); "
                        "frac_of_ncu_tf32_peak and useful_gemm_tflops (8 M^4 NT per stage and solve) beside it",
                "frac_of_ncu_tf32_peak": kd["tensor_frac_of_ncu_tf32_peak"],
                "useful_gemm_tflops": kd["useful_gemm_tflops"]}
    elif kd["roofline_bound"] == "fp32":
        roof = {"bound": "fp32", "kernel": names[dom], "achieved": kd["achieved_tflops"], "peak": fpeak,
                "unit": "TFLOP/s", "frac": kd["fp32_frac"],
                "peak_source": "nominal FP32 (148 SMs x 128 lanes x 2 x max SM clock); MEASURED_PEAKS.json has "
                               "no FP32 figure",
                "alg_flops_per_launch": kd["alg_flops_per_launch"],
                "hbm_frac": kd["frac"], "hbm_peak_gbs": peak}
    else:
        roof = {"bound": "hbm", "kernel": names[dom], "achieved": kd["achieved_gbs"], "peak": peak,
                "unit": "GB/s", "frac": kd["frac"],
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"}
    roof.update({"traffic": traffic_solve * args.batch if traffic_solve else None,
                 "alg_bytes_per_launch": kd["alg_bytes_per_launch"],
                 "fp32_peak_tflops": fpeak, "kernels": kernels})

    # the CPU baseline: the reference's solver on the host cores (rank 0, N=1 only), and
    # both precisions against its output after a few steps
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_accuracy:
        cs = args.cpu_steps
        keep = args.batch - 1
        r = run_reference_cpu(args.workload, args.batch, cs, args.order, args.peak_w, keep=keep)
        cpu_value = r["procs"] * M * NT * cs / r["max_seconds"]
        cpu = {"value": cpu_value, "unit": METRIC, "cores": r["procs"] * r["effective_omp_threads"],
               "kind": "reference",
               "sample": f"{r['procs']} concurrent reference solves of this workload (oracle/_ref, "
                         f"unmodified reference sources + FFTW-API shim), members {r['members'][-1]}.."
                         f"{r['members'][0]}, {cs} RK steps each"}
        if acc is not None and r["kept_output"] is not None:
            pk = make_problem(args.workload, keep, args.order, args.peak_w)
            for name, fl in (("fp32", 0), ("fp64", capi.MMP_F_FP64)):
                with mmp.Solver(pk.replace(flags=fl)) as s:
                    s.propagate(cs)
                    out = s.result()
                acc[f"relL2_max_{name}_vs_reference_member{keep}_{cs}_steps"] = float(
                    rel_l2_modes(out, r["kept_output"]).max())
    batch.close()
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": dist.world, "steps": K,
        "warmup": args.warmup, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.fp64 else "f32", "data": "synthetic",
        "config": workload_config(args, probe, dist.world),
        "state_mb_per_gpu": round(state_mb, 1), "kernels_chosen": chosen,
        "roofline": roof, "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
                "rk_steps_per_e2e_step": nsteps,
                "note": "one e2e step = set_fields (pinned H2D) + a solve of rk_steps_per_e2e_step steps + "
                        "get_result (D2H) for every batch member, wall clock"},
        "gpu_launches": int(launches), "clocks": clk, "accuracy": acc,
    }
    return line


def _play_stream(sv, stream, handles, keep=()):
    """Submit `stream` at its arrival times from a thread, wait for every request in
    order; returns (infos, outputs of the `keep` indices, makespan s)."""
    import threading
    ids = [None] * len(stream)

    def submitter():
        t0 = time.perf_counter()
        for i, (arr, p) in enumerate(stream):
            dt = arr - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            ids[i] = sv.submit(p, params=handles[i])

    th = threading.Thread(target=submitter)
    th.start()
    infos, outs = [None] * len(stream), {}
    for i in range(len(stream)):
        while ids[i] is None:
            time.sleep(0.001)
        out, infos[i] = sv.wait(ids[i], timeout=3600)
        if i in keep:
            outs[i] = out
    th.join()
    first = min(x["submit_s"] for x in infos)
    last = max(x["done_s"] for x in infos)
    return infos, outs, last - first


def _latency(infos):
    import numpy as np
    lat = np.array([x["done_s"] - x["submit_s"] for x in infos])
    return {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
            "mean": float(lat.mean()), "max": float(lat.max())}


def serve_arm(args, dist):
    """The mixed request stream through the serving loop (mmp_server_*): requests are
    submitted at their Poisson arrival times from host memory and waited for; the
    value is the stream's total M*NT*n_steps over the makespan (first arrival to last
    result, the server's clock), latency = result time - arrival time. The stream at
    200/s offers far more work than one GPU delivers, so its latencies are queueing
    time; a second, shorter stream at 0.7 of the capacity measured on the first shows
    the latency the continuous-batching loop itself adds."""
    import numpy as np
    import mm_propagation_b200 as mmp
    from mm_propagation_b200 import capi, workloads as W

    lib = mmp.lib()
    stream = W.stream(seed=1000 + dist.rank, n=args.requests, rate_hz=args.rate)
    handles = [p.to_params() for _, p in stream]          # host-side conversion, before timing
    work = sum(p.n_modes * p.nt * p.n_steps for _, p in stream)
    h2d = sum(p.n_modes * p.nt * 16 for _, p in stream)
    sv = mmp.Server()
    # warm-up: one short request per kernel shape (first-use costs: tables, graph capture)
    shapes = {}
    for _, p in stream:
        shapes.setdefault((p.nt, p.method_order), p)
    nw = max(args.warmup, 3)  # same step length, nw steps
    warm = [sv.submit(p.replace(n_steps=nw, fiber_length=p.fiber_length * nw / p.n_steps))
            for p in shapes.values()]
    for rid in warm:
        sv.wait(rid, timeout=600)
    # a seeded sample of requests, re-solved in FP64 after the stream for relL2
    check = set(np.random.default_rng(7).choice(len(stream), size=min(args.check, len(stream)),
                                                replace=False).tolist())
    clocks = Clocks(dist.local)
    dist.barrier()
    clocks.start()
    l0 = lib.mmp_kernel_launch_count()
    infos, outs, makespan = _play_stream(sv, stream, handles, check)
    launches = lib.mmp_kernel_launch_count() - l0
    clk = clocks.stop()
    makespan = dist.max(makespan)
    value = dist.world * work / makespan
    # below capacity: the same mix at 0.7 of the measured capacity (requests per second)
    sub = None
    capacity_rps = value / dist.world / (work / len(stream))
    sub_rate = 0.7 * capacity_rps if args.sub_rate is None else args.sub_rate
    if sub_rate > 0:
        n_sub = max(16, args.requests // 4)
        sub_stream = W.stream(seed=2000 + dist.rank, n=n_sub, rate_hz=sub_rate)
        sub_handles = [p.to_params() for _, p in sub_stream]
        sub_work = sum(p.n_modes * p.nt * p.n_steps for _, p in sub_stream)
        dist.barrier()
        sub_infos, _, sub_span = _play_stream(sv, sub_stream, sub_handles)
        sub_span = dist.max(sub_span)
        sub = {"rate_hz": sub_rate, "requests": n_sub, "offered_load_of_capacity": sub_rate / capacity_rps,
               "capacity_requests_per_s": capacity_rps, "latency_s": _latency(sub_infos),
               "value": dist.world * sub_work / sub_span,
               "service_s": _latency([{"submit_s": x["start_s"], "done_s": x["done_s"]} for x in sub_infos]),
               "note": "the same request mix (workloads.stream, another seed) at a Poisson rate below the "
                       "GPU's capacity: latency is admission + the solve sharing the GPU with its neighbours"}
    sv.close()
    acc = None
    if dist.rank == 0 and not args.no_accuracy:
        errs, work64, t64 = [], 0, 0.0
        for i in check:
            p = stream[i][1]
            with mmp.Solver(p.replace(flags=capi.MMP_F_FP64)) as s:
                t = time.perf_counter()
                s.propagate(p.n_steps)
                ref = s.result()  # synchronises: propagate + getResult, one FP64 solve on its own
                t64 += time.perf_counter() - t
            work64 += p.n_modes * p.nt * p.n_steps
            errs.append(float(rel_l2_modes(outs[i], ref).max()))
        acc = {"relL2_max_served_fp32_vs_fp64": max(errs), "checked_requests": len(check),
               "tolerance": 1e-5,
               # the same requests as plain single FP64 solves, one after another (wall clock)
               "fp64_single_solve_mode_samples_steps_per_s": work64 / t64}
    shapes_n = len({(p.nt, p.method_order) for _, p in stream})
    return {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": dist.world, "steps": 1,
        "warmup": len(warm), "ms_per_step": 1000.0 * makespan, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"serve: {args.requests} requests, Poisson arrivals at {args.rate}/s, "
                               "M in {1,3,6,10}, NT 2^11..2^15, L U(0.05,2) m, n_steps U(500,8000), "
                               "order 4/6, GRIN Q, Raman on (workloads.stream)",
                   "kernel_shapes": shapes_n, "total_mode_samples_steps": work,
                   "parallelism": f"replicas x{dist.world}", "l2": "inputs larger than L2"},
        "latency_s": _latency(infos),
        "sub_capacity": sub,
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
                "note": "one step = the whole stream: submit from host memory, propagate, result to host"},
        "gpu_launches": int(launches), "clocks": clk, "accuracy": acc,
    }


def batch_tableau(order):
    """Tableau coefficients from the library (mmp_tableau) for the byte model."""
    import mm_propagation_b200 as mmp
    a, b, c = mmp.tableau(order)
    a = [row + [0.0] * (len(b) - len(row)) for row in a]
    return a, b, c, len(b)


def main():
    args = parse()
    dist = Dist()
    try:
        if args.impl == "reference":
            line = reference_arm(args, dist)
        elif args.workload == "serve":
            line = serve_arm(args, dist)
        else:
            line = ours_arm(args, dist)
        if line is not None and dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
