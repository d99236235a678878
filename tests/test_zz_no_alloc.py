"""pdlpx_row_violation_noalloc -- the row-violation reduction for callers that
cannot allocate device memory (for example code running inside another
framework's memory pool).  The caller owns every device buffer; the entry point
keeps its block partials in a fixed device array instead of calling cudaMalloc.

Checked against the allocating entry point pdlpx_row_violation on two calls in
a row (different points, so the second call sees the first call's leftovers in
the shared array).  Both entry points pick the same threads per row and run
the same kernels in the same order, so the results must be identical to the
last bit.  Also covered: a smaller call after a larger one (fewer blocks than
the partials left in the array), the largest accepted size (exactly 4096
blocks) and the smallest rejected one, and m = 0.  This file is collected last
so that a failing run that stops at the first failure has already run every
other test.
"""
import numpy as np
import pytest

from mipx_b200 import _capi
from mipx_b200.pdlp import SparseMatrix, row_violation

pytestmark = pytest.mark.gpu


def _matrix(rows, cols, seed, max_len=30):
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, max_len, rows)
    rp = np.zeros(rows + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(cols, size=k, replace=False)) for k in lens])
    return SparseMatrix(rows, cols, values=rng.standard_normal(int(rp[-1])), col_indices=ci.astype(np.int32),
                        row_starts=rp.astype(np.int32))


def _bounds(ax, rng):
    rows = ax.size
    rl = np.where(np.arange(rows) % 4 == 0, -np.inf, ax - rng.random(rows))
    ru = np.where(np.arange(rows) % 4 == 1, np.inf, ax - 0.5 + rng.random(rows))
    return rl, ru


def _noalloc(lib, A, x, rl, ru, torch):
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (A.row_starts, A.col_indices, A.values, x, rl, ru)]
    d_out = torch.full((2,), -1.0, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    code = lib.pdlpx_row_violation_noalloc(A.rows, A.cols, A.numNonzeros(), *(a.data_ptr() for a in t),
                                           d_out.data_ptr(), None)
    torch.cuda.synchronize()
    return code, d_out.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    import torch

    lib = _capi.load()
    rng = np.random.default_rng(12)
    # a large call, then a smaller one: the second uses fewer blocks than the
    # partials the first left in the shared array
    for call, (rows, cols, seed) in enumerate([(5000, 3000, 11), (1200, 800, 13)]):
        A = _matrix(rows, cols, seed)
        x = rng.standard_normal(cols) * (1.0 + call)
        rl, ru = _bounds(A.multiply(x), rng)
        code, got = _noalloc(lib, A, x, rl, ru, torch)
        assert code == 0, lib.pdlpx_last_error(None)
        s_ref, mx_ref = row_violation(A, x, rl, ru)
        assert got[0] == s_ref and got[1] == mx_ref, (call, got, s_ref, mx_ref)


def test_noalloc_size_limit_is_exact():
    import torch

    lib = _capi.load()
    rng = np.random.default_rng(3)
    # one nonzero per row: one thread per row, so m rows need ceil(m / 256) blocks
    for rows, accepted in ((4096 * 256, True), (4096 * 256 + 1, False)):
        cols = 64
        ci = rng.integers(0, cols, rows).astype(np.int32)
        A = SparseMatrix(rows, cols, values=rng.standard_normal(rows), col_indices=ci,
                         row_starts=np.arange(rows + 1, dtype=np.int32))
        x = rng.standard_normal(cols)
        rl, ru = _bounds(A.values * x[ci], rng)  # one entry per row: A x elementwise
        code, got = _noalloc(lib, A, x, rl, ru, torch)
        if accepted:
            assert code == 0, lib.pdlpx_last_error(None)
            s_ref, mx_ref = row_violation(A, x, rl, ru)
            assert got[0] == s_ref and got[1] == mx_ref
        else:
            assert code == 1
            assert b"4096" in lib.pdlpx_last_error(None)
            assert got[0] == -1.0 and got[1] == -1.0  # nothing written


def test_noalloc_empty_rows_write_zero():
    import torch

    lib = _capi.load()
    A = SparseMatrix(0, 5, values=np.zeros(0), col_indices=np.zeros(0, np.int32), row_starts=np.zeros(1, np.int32))
    code, got = _noalloc(lib, A, np.ones(5), np.zeros(0), np.zeros(0), torch)
    assert code == 0, lib.pdlpx_last_error(None)
    assert got[0] == 0.0 and got[1] == 0.0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = _capi.load()
    # 2,000,000 one-nonzero rows need 7,813 blocks of 256 threads; the fixed scratch holds 4,096.
    # Rejected before any device pointer is touched.
    code = lib.pdlpx_row_violation_noalloc(2_000_000, 10, 2_000_000, 1, 1, 1, 1, 1, 1, 1, None)
    assert code == 1
    assert b"4096" in lib.pdlpx_last_error(None)
