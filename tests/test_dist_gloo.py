"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (one process per
rank, 127.0.0.1 rendezvous) check the timing reduction (max over ranks), the
whole-job aggregate (units of all ranks over the slowest rank's time) and the
barrier, the parts a torchrun launch of the bench uses around its GPU work."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    r, w, local, pg = bench.dist_init(world, backend="gloo")
    try:
        bench.barrier(pg)
        mx = bench.max_over_ranks(pg, float(rank + 1))
        sm = bench.sum_over_ranks(pg, 10.0 * (rank + 1))
        value, t = bench.aggregate(pg, 100.0 * (rank + 1), 2.0 + rank)
        q.put((r, w, mx, sm, value, t))
    finally:
        pg.destroy_process_group()


def test_two_gloo_ranks():
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    q = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for r, w, mx, sm, value, t in got:
        assert w == 2
        assert mx == 2.0          # max over ranks
        assert sm == 30.0         # 10 + 20
        assert t == 3.0           # the slowest rank's time
        assert value == 100.0     # (100 + 200) units / 3 s
