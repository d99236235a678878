"""Sharding of independent LPs across devices (host logic, no GPU):
pdlpx_shard_lps (longest-processing-time bin packing used by
pdlpx_batch_solve_devices) and bench.py's per-rank share of the batch."""
import sys
from pathlib import Path

import numpy as np
import pytest

from mipx_b200 import generators as G
from mipx_b200.pdlp import shard_lps

ROOT = Path(__file__).resolve().parents[1]


def _lpt_reference(w, ndev):
    """Plain-Python restatement of the rule: heaviest first (stable), each onto
    the least-loaded device, ties to the lower device index."""
    order = sorted(range(len(w)), key=lambda k: -w[k])
    load = [0] * ndev
    out = [0] * len(w)
    for k in order:
        d = min(range(ndev), key=lambda i: (load[i], i))
        out[k] = d
        load[d] += w[k]
    return out


@pytest.mark.parametrize("ndev", [1, 2, 3, 4, 8])
def test_shard_matches_rule_and_is_balanced(ndev):
    sizes = G.batch_sizes(512, seed=5)
    # per-iteration work of the batched workload's LPs: nnz ~ 8 n, plus m + n
    w = [int(8 * n + m + n) for m, n in sizes]
    got = shard_lps(w, ndev)
    assert list(got) == _lpt_reference(w, ndev)
    assert np.array_equal(got, shard_lps(w, ndev))  # deterministic
    loads = np.array([sum(w[k] for k in range(len(w)) if got[k] == d) for d in range(ndev)])
    assert loads.max() - loads.min() <= max(w)
    if ndev > 1:
        assert loads.max() / loads.mean() < 1.01  # 512 LPs spread to within 1%


def test_shard_edge_cases():
    assert list(shard_lps([], 4)) == []
    assert list(shard_lps([5], 4)) == [0]
    assert list(shard_lps([3, 3, 3, 3], 2)) == [0, 1, 0, 1]
    assert list(shard_lps([0, 0, 7], 3)) == [1, 1, 0]  # zero weight adds no load
    from mipx_b200._capi import PdlpxError
    with pytest.raises(PdlpxError):
        shard_lps([1, -1], 2)
    with pytest.raises(PdlpxError):
        shard_lps([1, 2], 0)


def test_bench_rank_lps_balances_work_and_covers_every_lp_once():
    """bench.py's batch line under torchrun: every LP on exactly one rank, and the
    ranks' shares of work (m + 9 n) within 1 % of each other on the 512-LP
    workload (its lognormal sizes make equal LP counts uneven in work)."""
    sys.path.insert(0, str(ROOT))
    import bench
    from mipx_b200 import generators as G
    sizes = G.batch_sizes(512, seed=5)
    for world in (1, 2, 4, 8):
        shares = [bench.rank_lps(sizes, r, world) for r in range(world)]
        assert sorted(k for s in shares for k in s) == list(range(len(sizes)))
        work = [sum(sizes[k][0] + 9 * sizes[k][1] for k in s) for s in shares]
        assert max(work) <= 1.01 * min(work), work
