"""The multi-GPU plumbing of bench.py (replicas: no data-path collective), run as two
gloo ranks on CPU: barrier, max over ranks of the timings, distinct per-rank work."""
import multiprocessing as mp
import os
import socket
import sys
from types import SimpleNamespace

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), MMP_DIST_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    try:
        d.barrier()
        m = d.max(10.0 * (rank + 1))
        args = SimpleNamespace(workload="grin2", order=4, peak_w=None, fp64=False, batch=3)
        probs = bench.make_batch_problems(args, d.rank)
        q.put((rank, m, [p.seed for p in probs]))
    finally:
        d.close()


def test_two_gloo_ranks_max_and_disjoint_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]           # max over ranks on every rank
    assert not set(res[0][2]) & set(res[1][2])            # each rank solves its own members
