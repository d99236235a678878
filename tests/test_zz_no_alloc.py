"""pdlpx_row_violation_noalloc -- the row-violation reduction for callers that
cannot allocate device memory (for example code running inside another
framework's memory pool).  The caller owns every device buffer; the entry point
keeps its block partials in a fixed device array instead of calling cudaMalloc.

Checked against the allocating entry point pdlpx_row_violation on two calls in
a row (different points, so the second call sees the first call's leftovers in
the shared array), within the tolerance the other row-violation tests use
(1e-12 relative).  This file is collected last so that a failing run that stops
at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from mipx_b200 import _capi
from mipx_b200.pdlp import SparseMatrix, row_violation

pytestmark = pytest.mark.gpu


def _matrix(rows, cols, seed):
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 30, rows)
    rp = np.zeros(rows + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(cols, size=k, replace=False)) for k in lens])
    return SparseMatrix(rows, cols, values=rng.standard_normal(int(rp[-1])), col_indices=ci.astype(np.int32),
                        row_starts=rp.astype(np.int32))


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    import torch

    lib = _capi.load()
    rows, cols = 5000, 3000
    A = _matrix(rows, cols, 11)
    dev = torch.device("cuda", 0)
    d_rp = torch.from_numpy(A.row_starts).to(dev)
    d_ci = torch.from_numpy(A.col_indices).to(dev)
    d_v = torch.from_numpy(A.values).to(dev)
    d_out = torch.full((2,), -1.0, dtype=torch.float64, device=dev)
    rng = np.random.default_rng(12)
    for call in range(2):
        x = rng.standard_normal(cols) * (1.0 + call)
        ax = A.multiply(x)
        rl = np.where(np.arange(rows) % 4 == 0, -np.inf, ax - rng.random(rows))
        ru = np.where(np.arange(rows) % 4 == 1, np.inf, ax - 0.5 + rng.random(rows))
        d_x = torch.from_numpy(x).to(dev)
        d_rl = torch.from_numpy(rl).to(dev)
        d_ru = torch.from_numpy(ru).to(dev)
        torch.cuda.synchronize()
        code = lib.pdlpx_row_violation_noalloc(rows, cols, A.numNonzeros(), d_rp.data_ptr(), d_ci.data_ptr(),
                                               d_v.data_ptr(), d_x.data_ptr(), d_rl.data_ptr(), d_ru.data_ptr(),
                                               d_out.data_ptr(), None)
        assert code == 0, lib.pdlpx_last_error(None)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        s_ref, mx_ref = row_violation(A, x, rl, ru)
        assert abs(got[0] - s_ref) <= 1e-12 * (1.0 + abs(s_ref)), (call, got, s_ref)
        assert abs(got[1] - mx_ref) <= 1e-12 * (1.0 + abs(mx_ref)), (call, got, mx_ref)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = _capi.load()
    # 2,000,000 one-nonzero rows need 7,813 blocks of 256 threads; the fixed scratch holds 4,096.
    # Rejected before any device pointer is touched.
    code = lib.pdlpx_row_violation_noalloc(2_000_000, 10, 2_000_000, 1, 1, 1, 1, 1, 1, 1, None)
    assert code == 1
    assert b"4096" in lib.pdlpx_last_error(None)
