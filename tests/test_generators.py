"""Seeded generators: deterministic, the stated shapes, and feasible by construction."""
import numpy as np

from mipx_b200 import generators as G


def _ax(lp, x):
    m = lp.matrix
    return np.add.reduceat(m.values * x[m.col_indices], m.row_starts[:-1]) * (np.diff(m.row_starts) > 0)


def test_random_lp_shape_and_feasibility():
    lp, x0 = G.random_lp(2000, 5000, 4, 12, 1)
    a, b = G.random_lp(2000, 5000, 4, 12, 1)[0], G.random_lp(2000, 5000, 4, 12, 2)[0]
    np.testing.assert_array_equal(lp.matrix.values, a.matrix.values)
    assert not np.array_equal(lp.obj, b.obj)
    assert lp.num_rows == 2000 and lp.num_cols == 5000
    per_col = np.bincount(lp.matrix.col_indices, minlength=5000)
    assert per_col.max() <= 12 and 35000 < lp.matrix.numNonzeros() < 45000
    ax = _ax(lp, x0)
    assert np.all(ax <= lp.row_upper + 1e-9) and np.all(ax >= lp.row_lower - 1e-9)
    eq = lp.row_lower == lp.row_upper
    assert eq.sum() == 1000
    assert np.all((x0 >= 0) & (x0 <= 10))
    rs = lp.matrix.row_starts
    for i in range(0, 2000, 97):
        seg = lp.matrix.col_indices[rs[i]:rs[i + 1]]
        assert np.all(np.diff(seg) > 0)


def test_transport_lp():
    lp, x0 = G.transport_lp(1000, 1000, 7)
    assert (lp.num_rows, lp.num_cols, lp.matrix.numNonzeros()) == (2000, 1_000_000, 2_000_000)
    assert np.all(lp.matrix.values == 1.0)
    supply = lp.row_upper[:1000]
    demand = lp.row_lower[1000:]
    assert np.all((supply >= 50) & (supply <= 150))
    assert abs(demand.sum() - 0.95 * supply.sum()) < 1e-6 * supply.sum()
    assert np.all((lp.obj >= 1) & (lp.obj <= 100))
    ax = _ax(lp, x0)
    assert np.all(ax[:1000] <= supply + 1e-9) and np.all(ax[1000:] >= demand - 1e-9)


def test_powerlaw_lp_small():
    lp, x0 = G.powerlaw_lp(5000, 20000, 2, 2000, 10.0, 0.01, 1e3, 11)
    counts = np.bincount(lp.matrix.col_indices, minlength=lp.num_cols)
    assert abs(counts.mean() - 10.0) < 1.0
    assert counts.max() <= 2000
    ax = _ax(lp, x0)
    assert np.all(ax <= lp.row_upper + 1e-6 * (1 + np.abs(lp.row_upper)))
    big = np.abs(lp.matrix.values).max()
    assert big > 100.0  # rows scaled by 1e3 exist


def test_batch_sizes():
    sizes = G.batch_sizes(512)
    ms = np.array([m for m, _ in sizes])
    assert len(sizes) == 512 and ms.min() >= 200 and ms.max() <= 20000
    assert 1200 < np.median(ms) < 1800
    assert all(n == round(2.5 * m) for m, n in sizes)


def test_oracle_library_generates_the_same_workloads():
    """The CPU-baseline legs build their inputs through the oracle library (so
    they never load the engine); its generators must give the engine's arrays
    exactly."""
    from oracle import oracle

    lib = oracle.gen_lib()
    cases = [(G.random_lp, (700, 1750, 4, 12, 9)), (G.transport_lp, (60, 80, 7)),
             (G.powerlaw_lp, (3000, 12000, 2, 2000, 10.0, 0.01, 1e3, 11))]
    for fn, args in cases:
        (a, xa), (b, xb) = fn(*args), fn(*args, lib=lib)
        for f in ("obj", "col_lower", "col_upper", "row_lower", "row_upper"):
            np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
        np.testing.assert_array_equal(a.matrix.row_starts, b.matrix.row_starts)
        np.testing.assert_array_equal(a.matrix.col_indices, b.matrix.col_indices)
        np.testing.assert_array_equal(a.matrix.values, b.matrix.values)
        np.testing.assert_array_equal(xa, xb)
