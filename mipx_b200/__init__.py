"""mipx_b200 -- B200-native PDLP engine, a drop-in for mipx's PDLP path.

The product is the C-ABI library ``_lib/libpdlpx.so`` (include/pdlpx.h) built
from ``csrc/`` for sm_100a; this package is its Python host side, mirroring
mipx's ``PdlpSolver`` / ``PdlpOptions`` / ``LpProblem`` interface.
"""
from .pdlp import (  # noqa: F401
    BasisStatus,
    LpProblem,
    LpResult,
    PdlpOptimalityNorm,
    PdlpOptions,
    PdlpSolver,
    Precision,
    Sense,
    SparseMatrix,
    Status,
    StopFlag,
    batch_solve,
    csr_spmv,
    kInf,
    read_mps,
    shard_lps,
    solve_mps,
)

__all__ = [
    "BasisStatus", "LpProblem", "LpResult", "PdlpOptimalityNorm", "PdlpOptions", "PdlpSolver", "Precision",
    "Sense", "SparseMatrix", "Status", "StopFlag", "batch_solve", "csr_spmv", "kInf", "read_mps", "shard_lps",
    "solve_mps",
]
