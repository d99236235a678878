"""TEST INFRASTRUCTURE: print mipx's src/lp/pdlp.cpp with the body of
PdlpSolver::solveGpu() replaced by the pdlpx binding (include/pdlpx_solvegpu.inc),
for `make -C oracle ref_bound`, which compiles the output from standard input
(nothing is written next to the reference or into the repository).

The replaced span runs from the definition line of solveGpu to the last
closing brace before the `#endif  // MIPX_HAS_CUDA` that ends the GPU block;
anything else in pdlp.cpp is passed through unchanged.  The script fails
loudly when the file does not have that shape.

    python oracle/bind_solvegpu.py <mipx>/src/lp/pdlp.cpp | g++ -x c++ -c - ...
"""
import sys
from pathlib import Path


def bind(text: str) -> str:
    lines = text.splitlines()
    head = "LpResult PdlpSolver::solveGpu() {"
    starts = [k for k, s in enumerate(lines) if s.strip() == head]
    if len(starts) != 1:
        raise SystemExit(f"expected one definition of PdlpSolver::solveGpu, found {len(starts)}")
    s0 = starts[0]
    ends = [k for k in range(s0 + 1, len(lines)) if lines[k].startswith("#endif") and "MIPX_HAS_CUDA" in lines[k]]
    if not ends:
        raise SystemExit("no '#endif  // MIPX_HAS_CUDA' after solveGpu")
    e = ends[0]
    close = max(k for k in range(s0 + 1, e) if lines[k].rstrip() == "}")
    out = lines[:s0] + ['#include "pdlpx_solvegpu.inc"'] + lines[close + 1:]
    return "\n".join(out) + "\n"


if __name__ == "__main__":
    sys.stdout.write(bind(Path(sys.argv[1]).read_text()))
