"""Benchmark of the PDLP path on B200.

Headline workload: the large single LP -- 500,000 rows x 2,000,000 columns,
column lengths power-law (2 to 2,000, mean 10; 20,130,372 nonzeros), values
N(0,1) with 1% of the rows scaled by 1e3, feasible by construction (seed 11)
-- solved to 1e-6 relative KKT (primal, dual and gap tolerances 1e-6), mixed
precision (FP32 matrix and SpMV, FP64 current iterates, checks, restarts and
polish).  One step = one full solve.  Metric: PDLP iterations per second; the
per-iteration working set (~420 MB) is far larger than the 126 MB L2.

* ``value``: iterations/s with the LP resident in HBM (the engine keeps its
  device image across solves), timed with CUDA events on the engine's stream
  (power iteration + restart cycles), after a 256 MiB L2-evicting write.
* ``e2e``: the same metric through the public API with host buffers -- load
  (host scaling with device Ruiz passes, H2D copies inside the solve), solve,
  copy x and y back -- per step.
* ``roofline``: the dominant kernel -- the fused primal step (A^T y + the
  Halpern primal step; long columns in row chunks with y in shared memory,
  short columns sliced ELL) -- timed live inside the timed solves: the
  restart-cycle graph records CUDA events around one primal and one dual step
  of every cycle (a step's time covers all of its launches).  Algorithmic
  bytes per step are in ``step_kernels.bytes`` (``step_bytes``); ``traffic``
  is ncu's dram__bytes_read.sum + dram__bytes_write.sum of the step's launches
  (profiles/).
* ``cpu_baseline`` and ``--impl reference``: the reference's own CPU
  PdlpSolver (compiled from its sources into oracle/_ref) on one host core --
  the reference PDLP is single-threaded per LP -- timed as the marginal rate
  between a 4- and a 12-iteration solve of the loaded LP (its load, i.e. its
  scaling pipeline, runs once; its power iteration is capped at 2 iterations
  for these samples, since its uncapped 5,000-iteration estimate takes about
  two minutes per solve on this LP and is not PDHG work).

Beside the headline (same JSON line, extra keys):
* ``transport``: the transportation LP, 1,000 x 1,000 (1M variables, 2,000
  rows, 2M unit nonzeros, seed 7): iterations/s, e2e, objective error against
  the stored HiGHS optimum, the reference's cuSPARSE FP64 GPU path (the plain
  FP64 GPU PDLP) and its CPU path as marginal rates.
* ``random_2000x5000``: the single random sparse LP the reference runs on CPU.
* ``batch``: 512 lognormal-sized random sparse LPs in one pdlpx_batch_solve
  call: LPs/s on the device and end to end, beside the engine's single-LP FP64
  mode, the reference's FP64 GPU path and the reference CPU path with one
  solver per host thread on samples of the same LPs.
* ``serving``: the request server on Poisson streams of branch-and-bound node
  LPs of a 20,000 x 50,000 base LP at several arrival rates.

With ``--gpus N`` under torchrun each rank solves its own replica of the large
LP (a single LP does not shard: replicas only); the batch is split across the
ranks (independent LPs, no collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

TOL = 1e-6
LARGE = dict(m=500_000, kmin=2, kmax=2000, kmean=10.0, big_frac=0.01, big_scale=1e3, seed=11)
WORKLOAD = ("power-law LP 500000 x 2000000 (20.1M nonzeros; column lengths 2-2000, mean 10; 1% of rows x1e3), "
            "to 1e-6 rel KKT")
METRIC = "PDLP iters/sec to 1e-6 rel KKT (power-law LP 500k x 2M)"
FLUSH_BYTES = 256 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--large-rows", type=int, default=LARGE["m"], help="rows of the headline LP (columns = 4 x rows)")
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-side", action="store_true", help="headline only (no transport / batch / serving lines)")
    p.add_argument("--no-transport", action="store_true")
    p.add_argument("--no-random", action="store_true")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--batch-lps", type=int, default=512)
    p.add_argument("--no-serving", action="store_true")
    p.add_argument("--serving-requests", type=int, default=512)
    p.add_argument("--serving-rates", default="5,20,200,2000",
                   help="arrival rates (requests/s) of the serving line; rates below the server's capacity "
                        "(~14 node LPs/s) send at most 128 requests")
    p.add_argument("--verbose", action="store_true")
    p.add_argument("--profile-large", type=int, default=0, metavar="M",
                   help="profiling run: one solve of an M x 4M power-law LP, no JSON line")
    p.add_argument("--profile-transport", action="store_true",
                   help="profiling run: the transportation LP, capped at --profile-iters")
    p.add_argument("--profile-batch", type=int, default=0, metavar="LPS",
                   help="profiling run: one pdlpx_batch_solve of the first LPS LPs of the batched workload")
    p.add_argument("--profile-family", type=int, default=0, metavar="LPS",
                   help="profiling run: LPS node LPs of the serving workload's base LP as one family pack")
    p.add_argument("--profile-iters", type=int, default=2000,
                   help="iteration cap of the --profile-* runs")
    p.add_argument("--profile-fp64", action="store_true",
                   help="profiling run of the single-LP cases in FP64 (the iterations after the hand-over)")
    return p.parse_args()


# ---------------------------------------------------------------------------
# multi-rank plumbing (one process per GPU)
# ---------------------------------------------------------------------------
def dist_init(n, backend=None):
    """One process per GPU (torchrun's RANK / WORLD_SIZE / LOCAL_RANK); NCCL on
    GPUs, gloo where none is visible (the multi-rank host logic on CPU)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return rank, world, local, pg


def _reduce(pg, value: float, op) -> float:
    if pg is None:
        return value
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(pg, value: float) -> float:
    return _reduce(pg, value, pg.ReduceOp.MAX if pg is not None else None)


def sum_over_ranks(pg, value: float) -> float:
    return _reduce(pg, value, pg.ReduceOp.SUM if pg is not None else None)


def aggregate(pg, units: float, seconds: float) -> tuple[float, float]:
    """Whole-job throughput of a weakly scaled run: the units every rank
    processed over the slowest rank's time (max over ranks, never wall clock)."""
    t = max_over_ranks(pg, seconds)
    return sum_over_ranks(pg, units) / t, t


def barrier(pg):
    import torch
    cuda = torch.cuda.is_available()
    if cuda:
        torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    if cuda:
        torch.cuda.synchronize()


def rank_lps(sizes, rank: int, world: int) -> list[int]:
    """The batch LPs (indices into `sizes`, (m, n) pairs) that rank `rank` of
    `world` solves: the engine's longest-processing-time sharding
    (pdlpx_shard_lps) on the per-iteration work m + n + 8 n of each LP (the
    generator draws 4-12 nonzeros per column), so the ranks' shares of work,
    not of LP counts, are balanced."""
    if world <= 1:
        return list(range(len(sizes)))
    from mipx_b200.pdlp import shard_lps
    owner = shard_lps([m + 9 * n for m, n in sizes], world)
    return [k for k in range(len(sizes)) if owner[k] == rank]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sms)}


def measured_peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


def ncu_traffic(kernel: str, workload_key: str):
    """Per-launch DRAM bytes of the kernel from the committed ncu summary, or None."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    try:
        return json.loads(p.read_text()).get(workload_key, {}).get(kernel)
    except ValueError:
        return None


# ---------------------------------------------------------------------------
# algorithmic bytes of the step kernels (per launch)
# ---------------------------------------------------------------------------
def step_bytes(m: int, n: int, nnz: int) -> dict:
    """Bytes a CSR implementation of each fused step must move once per launch.

    FP32 kernels (mixed phase): matrix values + indices 8 B/nnz, row pointers;
    primal: the FP32 copy of y_cur gathered once (4 m), per column the packed
    constants (16 B), x_cur read + write (FP64, 16 B), x_init (4 B), x_refl
    write (4 B); dual: x_refl gathered once (4 n), per row the packed
    constants (16 B), y_cur read + write (16 B), y_init (4 B), the FP32 copy of
    y_cur written (4 B).  (The tiled long-column launch stores its entries in
    6 B and adds per-chunk partial sums; the CSR figure is kept as the
    algorithmic one.)  FP64 kernels: 12 B/nnz, 32 B packs, FP64 anchors and
    reflections, y_cur gathered in FP64."""
    return {
        "primal_fp32": 4 * (n + 1) + 8 * nnz + 4 * m + 40 * n,
        "dual_fp32": 4 * (m + 1) + 8 * nnz + 4 * n + 40 * m,
        "primal_fp64": 4 * (n + 1) + 12 * nnz + 8 * m + 64 * n,
        "dual_fp64": 4 * (m + 1) + 12 * nnz + 8 * n + 56 * m,
    }


# ---------------------------------------------------------------------------
# baselines: the reference's own PdlpSolver (oracle/_ref), never the engine
# ---------------------------------------------------------------------------
def ref_marginal_rate(lp, lo: int, hi: int, sv_max_iter: int, reps: int = 1, gpu: bool = False,
                      warm: bool = False) -> dict:
    """Iterations/s of the reference PdlpSolver on `lp`: loaded once, then the
    wall time of a `hi`-iteration solve minus that of a `lo`-iteration solve
    (same power-iteration cap) over hi - lo; median over `reps` pairs.  With
    `warm`, one untimed `lo`-iteration solve runs first: the first solve pays
    the one-time costs (the GPU path's library handles and lazy kernel
    loading), which would otherwise shrink the difference and inflate the rate."""
    from mipx_b200.pdlp import PdlpOptions
    from oracle import oracle
    o = PdlpOptions(verbose=False, use_gpu=gpu, gpu_min_rows=0, gpu_min_nnz=0, primal_tol=TOL, dual_tol=TOL,
                    optimality_tol=TOL)
    rates, t_load = [], time.perf_counter()
    with oracle.RefSession(lp, o, gpu=gpu) as rs:
        t_load = time.perf_counter() - t_load
        if warm:
            rs.run(lo, sv_max_iter)
        for _ in range(reps):
            _, t0 = rs.run(lo, sv_max_iter)
            _, t1 = rs.run(hi, sv_max_iter)
            rates.append((hi - lo) / max(t1 - t0, 1e-9))
    return {"value": statistics.median(rates), "unit": "iters/s", "load_s": t_load,
            "sample": f"reference {'FP64 GPU (cuSPARSE)' if gpu else 'CPU'} PdlpSolver loaded once; marginal rate "
                      f"between {lo}- and {hi}-iteration solves, power iteration capped at {sv_max_iter}; "
                      f"median of {reps}{', after one untimed warm-up solve' if warm else ''}"}


def ref_solve_lps(lps, gpu: bool, threads: int = 1) -> dict:
    """LPs/s of the reference PdlpSolver solving `lps` to 1e-6 relative KKT:
    `threads` host threads, one solver each (the reference's solvers are
    independent per instance); GPU arm: one solver at a time on the device,
    after one untimed solve of the first LP (the one-time library set-up)."""
    from concurrent.futures import ThreadPoolExecutor

    from mipx_b200.pdlp import PdlpOptions
    from oracle import oracle
    o = PdlpOptions(verbose=False, use_gpu=gpu, gpu_min_rows=0, gpu_min_nnz=0, primal_tol=TOL, dual_tol=TOL,
                    optimality_tol=TOL, max_solve_seconds=120.0)
    if gpu and lps:
        oracle.ref_solve(lps[0], o, gpu=True)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:  # ctypes releases the GIL inside the solves
        out = list(ex.map(lambda lp: oracle.ref_solve(lp, o, gpu=gpu)[0], lps))
    wall = time.perf_counter() - t0
    return {"lps_per_sec": len(lps) / wall, "lps": len(lps), "threads": threads, "wall_s": wall,
            "optimal": sum(1 for r in out if int(r.status) == 0), "objectives": [r.objective for r in out],
            "iterations": [r.iterations for r in out]}


# ---------------------------------------------------------------------------
# engine workloads
# ---------------------------------------------------------------------------
def solve_steps(solver, steps: int, flush) -> dict:
    """`steps` full solves of the loaded LP, an L2-evicting write before each;
    device time from the engine's CUDA events."""
    import torch

    from mipx_b200.pdlp import Status
    out = {k: [] for k in ("iters", "fp64", "dev", "lat", "launches", "objs", "kkts")}
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        r = solver.solve()
        if r.status != Status.Optimal:
            raise RuntimeError(f"solve ended with status {r.status!r}")
        out["iters"].append(r.iterations)
        out["fp64"].append(r.fp64_iterations)
        out["dev"].append(r.device_seconds)
        out["lat"].append(r.solve_seconds)
        out["launches"].append(r.kernel_launches)
        out["objs"].append(r.objective)
        out["kkts"].append(max(r.rel_primal_resid, r.rel_dual_resid, r.rel_gap))
    return out


def e2e_steps(lp, opts, steps: int, flush) -> tuple[float, int]:
    """The metric through the public API with host buffers: a new solver per
    step, load (copies the caller's arrays, scales; H2D inside the solve),
    solve, read x and y back.  Returns (seconds, iterations)."""
    import torch

    from mipx_b200.pdlp import PdlpSolver
    t, it = 0.0, 0
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s = PdlpSolver()
        s.setOptions(opts)
        s.load(lp)
        r = s.solve()
        s.getPrimalValues()
        s.getDualValues()
        t += time.perf_counter() - t0
        it += r.iterations
        del s
    return t, it


def step_kernel_report(solver, m: int, n: int, nnz: int, peak: float) -> dict:
    """Live step-kernel times of the last solve against the algorithmic bytes."""
    from mipx_b200.pdlp import Precision
    b = step_bytes(m, n, nnz)
    out = {"bytes": b}
    for tag, prec in (("fp32", Precision.Mixed), ("fp64", Precision.FP64)):
        t = solver.stepTimes(prec)
        if t["samples"] <= 0:
            continue
        e = {"samples": t["samples"], "primal_us": 1e3 * t["primal_ms"], "dual_us": 1e3 * t["dual_ms"],
             "primal_GBps": b[f"primal_{tag}"] / (t["primal_ms"] * 1e-3) / 1e9,
             "dual_GBps": b[f"dual_{tag}"] / (t["dual_ms"] * 1e-3) / 1e9}
        e["primal_frac"] = e["primal_GBps"] / peak
        e["dual_frac"] = e["dual_GBps"] / peak
        out[tag] = e
    return out


def large_headline(args, rank, world, local, pg, flush) -> dict:
    from mipx_b200 import generators as G
    from mipx_b200.pdlp import PdlpOptions, PdlpSolver
    m = args.large_rows
    lp, _ = G.powerlaw_lp(m, 4 * m, LARGE["kmin"], LARGE["kmax"], LARGE["kmean"], LARGE["big_frac"],
                          LARGE["big_scale"], LARGE["seed"])
    n, nnz = lp.num_cols, lp.matrix.numNonzeros()
    opts = PdlpOptions(verbose=args.verbose, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL, device=local)
    solver = PdlpSolver()
    solver.setOptions(opts)
    t0 = time.perf_counter()
    solver.load(lp)
    load_s = time.perf_counter() - t0
    for _ in range(max(3, args.warmup)):
        solver.solve()
    barrier(pg)
    with ClockSampler(local) as clk:
        t_wall = time.perf_counter()
        res = solve_steps(solver, args.steps, flush)
        barrier(pg)
        wall = time.perf_counter() - t_wall
    value, t_dev = aggregate(pg, float(sum(res["iters"])), sum(res["dev"]))
    lps = sum_over_ranks(pg, float(args.steps)) / t_dev
    peak, peak_kind = measured_peak_hbm()
    kern = step_kernel_report(solver, m, n, nnz, peak)
    e2e_t, e2e_it = e2e_steps(lp, opts, max(1, args.e2e_steps), flush)
    e2e_t = max_over_ranks(pg, e2e_t)
    e2e_val = sum_over_ranks(pg, float(e2e_it)) / e2e_t
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = ref_marginal_rate(lp, 4, 12, 2)
            cpu.update(cores=1, kind="reference")
        except Exception as exc:  # the baseline is a report, never a reason to lose the line
            cpu = {"value": None, "error": str(exc)}
    return {"m": m, "n": n, "nnz": nnz, "res": res, "value": value, "t_dev": t_dev, "lps": lps, "wall": wall,
            "clk": clk.summary(), "peak": peak, "peak_kind": peak_kind, "kern": kern,
            "cfg": dict(solver.launchConfig(), long_tiles=solver.longTiles()),
            "e2e": e2e_val, "e2e_steps": max(1, args.e2e_steps), "cpu": cpu, "load_s": load_s,
            "h2d": int(sum(a.nbytes for a in lp.arrays())), "d2h": 8 * (n + m)}


def transport_line(local, flush) -> dict:
    from mipx_b200 import generators as G
    from mipx_b200.pdlp import PdlpOptions, PdlpSolver, Precision
    lp, _ = G.transport_lp(1000, 1000, 7)
    m, n, nnz = lp.num_rows, lp.num_cols, lp.matrix.numNonzeros()
    opts = PdlpOptions(verbose=False, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL, device=local)
    s = PdlpSolver()
    s.setOptions(opts)
    s.load(lp)
    s.solve()  # device image, graphs
    res = solve_steps(s, 2, flush)
    peak, _ = measured_peak_hbm()
    kern = step_kernel_report(s, m, n, nnz, peak)
    e2e_t, e2e_it = e2e_steps(lp, opts, 1, flush)
    gold = json.loads((ROOT / "tests" / "golden" / "ref_pdlp.json").read_text()).get("transport_1000x1000", {})
    hi = gold.get("highs_objective")
    obj = res["objs"][-1]
    out = {"workload": "transportation LP 1000 x 1000 (1M vars, 2k rows, 2M unit nonzeros, seed 7), to 1e-6 rel KKT",
           "iters_per_sec": sum(res["iters"]) / sum(res["dev"]), "e2e_iters_per_sec": e2e_it / e2e_t,
           "iterations": res["iters"][-1], "fp64_iterations": res["fp64"][-1], "device_s": res["dev"][-1],
           "objective": obj, "highs_objective": hi,
           "objective_rel_err_vs_highs": abs(obj - hi) / abs(hi) if hi else None, "max_rel_kkt": max(res["kkts"]),
           "step_kernels": kern, "config": s.launchConfig()}
    s64 = PdlpSolver()
    s64.setOptions(PdlpOptions(verbose=False, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL, device=local,
                               precision=Precision.FP64))
    s64.load(lp)
    r64 = s64.solve()
    out["engine_fp64_iters_per_sec"] = r64.iterations / r64.device_seconds
    try:  # the reference's own FP64 GPU path (cuSPARSE): the plain FP64 GPU PDLP
        g = ref_marginal_rate(lp, 1000, 3000, 5000, reps=3, gpu=True, warm=True)
        out["reference_fp64_gpu"] = g
        out["speedup_vs_reference_fp64_gpu"] = out["iters_per_sec"] / g["value"]
    except Exception as exc:
        out["reference_fp64_gpu"] = {"error": str(exc)}
    try:
        c = ref_marginal_rate(lp, 100, 300, 5000)
        c.update(cores=1, kind="reference")
        out["cpu_baseline"] = c
    except Exception as exc:
        out["cpu_baseline"] = {"error": str(exc)}
    return out


def random_line(local) -> dict:
    """The single 2,000 x 5,000 random sparse LP (seed 1), which the reference runs on CPU."""
    from mipx_b200 import generators as G
    from mipx_b200.pdlp import PdlpOptions, PdlpSolver
    from oracle import oracle
    lp, _ = G.random_lp(2000, 5000, 4, 12, 1)
    s = PdlpSolver()
    s.setOptions(PdlpOptions(verbose=False, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL, device=local))
    s.load(lp)
    s.solve()
    rs = [s.solve() for _ in range(3)]
    t0 = time.perf_counter()
    ref, _, _ = oracle.ref_solve(lp, PdlpOptions(verbose=False, use_gpu=False, primal_tol=TOL, dual_tol=TOL,
                                                 optimality_tol=TOL))
    t_ref = time.perf_counter() - t0
    obj = rs[-1].objective
    return {"workload": "random sparse LP 2000 x 5000 (4-12 nonzeros per column, seed 1), to 1e-6 rel KKT",
            "iters_per_sec": sum(r.iterations for r in rs) / sum(r.device_seconds for r in rs),
            "lps_per_sec": len(rs) / sum(r.device_seconds for r in rs),
            "iterations": rs[-1].iterations, "device_s": rs[-1].device_seconds, "objective": obj,
            "reference_objective": ref.objective,
            "objective_rel_err_vs_reference": abs(obj - ref.objective) / max(1.0, abs(ref.objective)),
            "cpu_baseline": {"value": ref.iterations / t_ref, "unit": "iters/s", "cores": 1, "kind": "reference",
                             "sample": f"one full reference CPU solve ({ref.iterations} iterations, load included)",
                             "lps_per_sec": 1.0 / t_ref}}


def batch_line(rank, world, local, count: int) -> dict:
    """The batched workload: `count` random sparse LPs of lognormal size (median
    1,500 rows, sigma 0.8, clipped to [200, 20,000], n = 2.5 m, 4-12 nonzeros
    per column, seeds 1000 + k) solved to 1e-6 relative KKT by one
    pdlpx_batch_solve call; under torchrun each rank solves its own share."""
    from mipx_b200 import generators as G
    from mipx_b200.pdlp import PdlpOptions, PdlpSolver, Precision, Status, batch_solve
    tol = dict(primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL, device=local)
    sizes = G.batch_sizes(count, seed=5)
    lps = [G.random_lp(sizes[k][0], sizes[k][1], 4, 12, 1000 + k)[0] for k in rank_lps(sizes, rank, world)]
    batch_solve(lps[:4], PdlpOptions(verbose=False, max_iter=400, **tol))  # warm-up (module load)
    t0 = time.perf_counter()
    out = batch_solve(lps, PdlpOptions(verbose=False, **tol))
    wall = time.perf_counter() - t0
    dev = out[0][0].device_seconds
    line = {"workload": f"{count} random sparse LPs, lognormal sizes (median m 1500, n = 2.5 m), to 1e-6 rel KKT, "
                        "one pdlpx_batch_solve call" + (f" per rank ({len(lps)} here)" if world > 1 else ""),
            "lps": len(lps), "nonzeros": sum(lp.matrix.numNonzeros() for lp in lps),
            "lps_per_sec": len(lps) / dev, "e2e_lps_per_sec": len(lps) / wall, "device_s": dev, "wall_s": wall,
            "optimal": sum(1 for r, _, _ in out if r.status == Status.Optimal),
            "iterations_total": int(sum(r.iterations for r, _, _ in out)),
            "iterations_max": int(max(r.iterations for r, _, _ in out))}
    if rank != 0:
        return line
    sample = list(range(16))
    single = 0.0
    for k in sample:  # the engine's single-LP FP64 mode
        s = PdlpSolver()
        s.setOptions(PdlpOptions(verbose=False, precision=Precision.FP64, **tol))
        s.load(lps[k])
        single += s.solve().device_seconds
    line["single_lp_fp64_lps_per_sec"] = len(sample) / single
    line["speedup_vs_single_lp_fp64"] = line["lps_per_sec"] / line["single_lp_fp64_lps_per_sec"]
    try:  # the reference's own FP64 GPU path, one LP at a time (it builds and frees its device state per solve)
        g = ref_solve_lps([lps[k] for k in sample], gpu=True)
        line["reference_fp64_gpu"] = {k: g[k] for k in ("lps_per_sec", "lps", "wall_s", "optimal")}
        line["speedup_vs_reference_fp64_gpu"] = line["lps_per_sec"] / g["lps_per_sec"]
    except Exception as exc:
        line["reference_fp64_gpu"] = {"error": str(exc)}
    try:  # the reference CPU path, one solver per host thread over a sample
        threads = os.cpu_count() or 1
        cpu_sample = list(range(min(len(lps), 2 * threads)))
        c = ref_solve_lps([lps[k] for k in cpu_sample], gpu=False, threads=threads)
        errs = [abs(out[k][0].objective - c["objectives"][i]) / max(1.0, abs(c["objectives"][i]))
                for i, k in enumerate(cpu_sample) if int(out[k][0].status) == 0]
        line["cpu_baseline"] = {"value": c["lps_per_sec"], "unit": "LPs/s", "cores": threads, "kind": "reference",
                                "sample": f"the first {len(cpu_sample)} LPs of the batch, reference CPU PdlpSolver, "
                                          f"one solver per host thread ({threads} threads)",
                                "optimal": c["optimal"]}
        line["objective_rel_err_vs_reference_max"] = max(errs) if errs else None
    except Exception as exc:
        line["cpu_baseline"] = {"error": str(exc)}
    return line


def serving_line(local, requests: int, rates) -> dict:
    """Branch-and-bound node LPs of a 20,000 x 50,000 random sparse base LP (4-12
    nonzeros per column, 30% of the columns marked integer; each node fixes
    1-5% of the integer columns to floor/ceil of x0 and appends 0-50 cuts of
    20-200 nonzeros) arriving as Poisson streams, each warm-started from the
    base request; latency is submit -> result."""
    from mipx_b200 import generators as G
    from mipx_b200.pdlp import PdlpOptions, PdlpSolver, Precision, Server, Status
    tol = dict(primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL, verbose=False, device=local)
    base, x0 = G.random_lp(20000, 50000, 4, 12, 101)
    ints = G.integer_marks(base.num_cols)
    nodes = [G.node_lp(base, x0, ints, 1000 + k) for k in range(requests)]
    out = {"workload": f"{requests} node LPs of a 20000 x 50000 base LP ({base.matrix.numNonzeros()} nonzeros) per "
                       "arrival rate, Poisson arrivals, warm-started from the base, to 1e-6 rel KKT; family packs "
                       "of up to 32 nodes, 4 packs in flight"}
    single = 0.0
    for nd in nodes[:4]:
        s = PdlpSolver()
        s.setOptions(PdlpOptions(precision=Precision.FP64, **tol))
        s.load(nd)
        single += s.solve().device_seconds
    out["single_lp_fp64_lps_per_sec"] = 4 / single
    out["single_lp_fp64_seconds_per_lp"] = single / 4
    for rate in rates:
        # below capacity a stream of 128 requests shows the unqueued latency
        # without stretching the run (512 requests at 5/s would take 100 s)
        count = requests if rate >= 20 else min(requests, 128)
        arrivals = np.cumsum(np.random.default_rng(7).exponential(1.0 / rate, count))
        with Server(PdlpOptions(**tol), max_packs=4, max_pack_lps=32, batch_window_ms=50) as srv:
            tb = srv.submit(base)
            srv.wait(tb)
            start = time.perf_counter()
            tickets = []
            for k, nd in enumerate(nodes[:count]):
                d = start + arrivals[k] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets.append(srv.submit(nd, warm=tb))
            res = [srv.wait(t)[0] for t in tickets]
            end = time.perf_counter()
            st = srv.stats()
        lps = count / (end - start)
        out[f"rate_{int(rate)}"] = {
            "offered_req_per_sec": rate, "requests": count, "p50_latency_s": st["p50_latency_s"],
            "p99_latency_s": st["p99_latency_s"],
            "lps_per_sec": lps, "optimal": sum(1 for r in res if r.status == Status.Optimal),
            "iterations_median": float(np.median([r.iterations for r in res])),
            "speedup_vs_single_lp_fp64": lps / out["single_lp_fp64_lps_per_sec"]}
    return out


def profile_run(args, local) -> None:
    """Capped runs for ncu (no JSON line)."""
    from mipx_b200 import generators as G
    from mipx_b200.pdlp import PdlpOptions, PdlpSolver, Precision, batch_solve
    o = PdlpOptions(verbose=False, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL, device=local,
                    max_iter=args.profile_iters)
    if args.profile_batch:
        sizes = G.batch_sizes(512, seed=5)[:args.profile_batch]
        lps = [G.random_lp(m, n, 4, 12, 1000 + k)[0] for k, (m, n) in enumerate(sizes)]
        out = batch_solve(lps, o)
        print(f"profile batch: {len(lps)} LPs, {sum(r.iterations for r, _, _ in out)} LP-iterations, "
              f"device {out[0][0].device_seconds:.3f}s, launches {out[0][0].kernel_launches}", flush=True)
    if args.profile_family:
        from mipx_b200.pdlp import Server
        base, x0 = G.random_lp(20000, 50000, 4, 12, 101)
        ints = G.integer_marks(base.num_cols)
        nodes = [G.node_lp(base, x0, ints, 1000 + k) for k in range(args.profile_family)]
        with Server(o, max_packs=1, max_pack_lps=32, batch_window_ms=2000) as srv:
            tb = srv.submit(base)
            srv.wait(tb)
            t0 = time.perf_counter()
            res = [srv.wait(t) for t in [srv.submit(nd, warm=tb) for nd in nodes]]
            wall = time.perf_counter() - t0
        print(f"profile family: {len(nodes)} node LPs, {sum(r.iterations for r, _, _ in res)} LP-iterations, "
              f"device {max(r.device_seconds for r, _, _ in res):.3f}s, wall {wall:.3f}s", flush=True)
    lps = []
    if args.profile_large:
        lps.append(G.powerlaw_lp(args.profile_large, 4 * args.profile_large, 2, 2000, 10.0, 0.01, 1e3, 11)[0])
    if args.profile_transport:
        lps.append(G.transport_lp(1000, 1000, 7)[0])
    if args.profile_fp64:
        o.precision = Precision.FP64
    for lp in lps:
        s = PdlpSolver()
        s.setOptions(o)
        s.load(lp)
        r = s.solve()
        print(f"profile: {lp.num_rows} x {lp.num_cols}, {lp.matrix.numNonzeros()} nnz, {r.iterations} iterations, "
              f"device {r.device_seconds:.3f}s, launches {r.kernel_launches}, config {s.launchConfig()}", flush=True)


def run_reference(args, rank, pg):
    """The reference's own CPU PdlpSolver (oracle/_ref, compiled from its
    sources) on the headline LP, rank 0 only.  Nothing here loads the engine
    library: the workload generator comes from the oracle library."""
    if rank != 0:
        return
    from mipx_b200 import generators as G
    from mipx_b200.pdlp import PdlpOptions
    from oracle import oracle
    m = args.large_rows
    lp, _ = G.powerlaw_lp(m, 4 * m, LARGE["kmin"], LARGE["kmax"], LARGE["kmean"], LARGE["big_frac"],
                          LARGE["big_scale"], LARGE["seed"], lib=oracle.gen_lib())
    o = PdlpOptions(verbose=False, use_gpu=False, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL)
    lo, hi, sv = 4, 12, 2
    vals = []
    with oracle.RefSession(lp, o) as rs:
        for _ in range(args.warmup):
            rs.run(lo, sv)
        for _ in range(max(1, args.steps)):
            _, t0 = rs.run(lo, sv)
            _, t1 = rs.run(hi, sv)
            vals.append((hi - lo) / max(t1 - t0, 1e-9))
    v = statistics.median(vals)
    sample = (f"reference CPU PdlpSolver (use_gpu=false) loaded once; per step the marginal rate between a {lo}- and "
              f"a {hi}-iteration solve, power iteration capped at {sv}; median over steps")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "iters/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * (hi - lo) / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, seed 11)",
            "config": {"workload": WORKLOAD, "m": lp.num_rows, "n": lp.num_cols, "nnz": lp.matrix.numNonzeros(),
                       "sample": sample},
            "cpu_baseline": {"value": v, "unit": "iters/s", "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local, pg = dist_init(args.gpus)
    if args.impl == "reference":
        run_reference(args, rank, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.profile_batch or args.profile_large or args.profile_family or args.profile_transport:
        profile_run(args, local)
        return
    import torch
    torch.cuda.set_device(local)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    H = large_headline(args, rank, world, local, pg, flush)
    res = H["res"]

    def side_line(skip, fn, *a):  # a report beside the headline, never a reason to lose the line
        if args.no_side or skip:
            return None
        try:
            return fn(*a)
        except Exception as exc:
            return {"error": str(exc)}

    transport = side_line(args.no_transport or world > 1, transport_line, local, flush)
    rnd = side_line(args.no_random or world > 1, random_line, local)
    batch = side_line(args.no_batch, batch_line, rank, world, local, args.batch_lps)
    if not (args.no_side or args.no_batch):
        # whole-job LPs/s of the batch over all ranks (every rank takes part, error or not)
        ok = batch is not None and "device_s" in batch
        agg, _ = aggregate(pg, float(batch["lps"]) if ok else 0.0, batch["device_s"] if ok else 1e-9)
        if ok:
            batch["job_lps_per_sec"] = agg
    rates = [float(r) for r in args.serving_rates.split(",") if r]
    serving = side_line(args.no_serving or world > 1, serving_line, local, args.serving_requests, rates)

    if rank == 0:
        kern = H["kern"]
        # the dominant kernel: the primal step in the precision that ran most iterations
        fp64_share = sum(res["fp64"]) / max(sum(res["iters"]), 1)
        tag = "fp64" if ("fp32" not in kern or (fp64_share > 0.5 and "fp64" in kern)) else "fp32"
        k = kern[tag]
        traffic = ncu_traffic(f"primal_{tag}", f"powerlaw_{H['m']}x{H['n']}")
        b = kern["bytes"]
        it32 = sum(res["iters"]) - sum(res["fp64"])
        solve_gbps = (it32 * (b["primal_fp32"] + b["dual_fp32"]) +
                      sum(res["fp64"]) * (b["primal_fp64"] + b["dual_fp64"])) / sum(res["dev"]) / 1e9
        line = {
            "metric": METRIC, "value": H["value"], "unit": "iters/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": 1000.0 * H["t_dev"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 (matrix, SpMV) + fp64 (current iterates, checks, restarts, polish)",
            "data": "synthetic (seeded generator, seed 11)",
            "config": {"workload": WORKLOAD, "m": H["m"], "n": H["n"], "nnz": H["nnz"], "tolerance": TOL,
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (~420 MB per iteration vs 126 MB); 256 MiB L2-evicting write "
                             "before each step", "launch": H["cfg"]},
            "iterations_per_solve": statistics.median(res["iters"]),
            "fp64_iterations_per_solve": statistics.median(res["fp64"]),
            "lps_per_sec": H["lps"],
            "latency_s": {"p50": float(np.percentile(res["lat"], 50)), "p99": float(np.percentile(res["lat"], 99))},
            "objective": res["objs"][-1], "max_rel_kkt": max(res["kkts"]), "wall_s": H["wall"], "load_s": H["load_s"],
            "clocks": H["clk"],
            "e2e": {"value": H["e2e"], "unit": "iters/s", "h2d_bytes_per_step": H["h2d"],
                    "d2h_bytes_per_step": H["d2h"], "steps": H["e2e_steps"]},
            "gpu_launches": int(sum(res["launches"])),
            "roofline": {"bound": "hbm",
                         "kernel": f"primal step, {tag.upper()} kernels (A^T y + Halpern step; long columns "
                                   + ("in row chunks with y in shared memory" if H["cfg"]["long_tiles"]["chunks"] else "CSR")
                                   + ", short columns sliced ELL)",
                         "achieved": k["primal_GBps"], "peak": H["peak"], "peak_kind": H["peak_kind"], "unit": "GB/s",
                         "frac": k["primal_frac"], "traffic": traffic, "algorithmic_bytes": b[f"primal_{tag}"],
                         "timing": "live: CUDA events around one primal and one dual step of every restart cycle of "
                                   "the timed solves (event-record nodes in the cycle graph)"},
            "step_kernels": kern,
            # whole-solve cross-check: algorithmic bytes of every iteration over the device time of the solves
            # (power iteration and check passes are in the time, not in the bytes)
            "solve_GBps": solve_gbps,
            "cpu_baseline": H["cpu"],
            "transport": transport,
            "random_2000x5000": rnd,
            "batch": batch,
            "serving": serving,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
