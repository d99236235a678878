// Exercise of the C++ mirror of mipx's PDLP interface (include/pdlpx.hpp).
//   pdlpx_api_test host   -- paths that never reach the device (defaults, not
//                            loaded, LPs without rows: closed form on the host)
//   pdlpx_api_test gpu    -- solves on the device
// Prints one line per check; exits non-zero on the first failure.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "pdlpx.hpp"

using pdlpx::kInf;
using pdlpx::LpProblem;
using pdlpx::PdlpSolver;
using pdlpx::Status;

static int fails = 0;
#define CHECK(cond)                                                  \
    do {                                                             \
        if (cond) {                                                  \
            std::printf("ok   %s\n", #cond);                         \
        } else {                                                     \
            std::printf("FAIL %s (line %d)\n", #cond, __LINE__);     \
            ++fails;                                                 \
        }                                                            \
    } while (0)

// min -x - y  s.t.  x + y <= 4,  x, y >= 0  -> -4 (test_pdlp.cpp buildSimpleLp)
static LpProblem simpleLp() {
    LpProblem lp;
    lp.num_cols = 2;
    lp.obj = {-1.0, -1.0};
    lp.col_lower = {0.0, 0.0};
    lp.col_upper = {kInf, kInf};
    lp.num_rows = 1;
    lp.row_lower = {-kInf};
    lp.row_upper = {4.0};
    lp.row_starts = {0, 2};
    lp.col_indices = {0, 1};
    lp.values = {1.0, 1.0};
    return lp;
}

static int host() {
    pdlpx::PdlpOptions o;
    CHECK(o.termination_eval_frequency == 200);
    CHECK(o.anderson_window_size == 5 && o.anderson_acceleration == 0);
    PdlpSolver s;
    o.verbose = 0;
    s.setOptions(o);
    CHECK(s.options().verbose == 0);
    CHECK(s.solve().status == Status::Error);  // not loaded (pdlp.cpp:802-805)
    LpProblem empty;
    empty.obj_offset = 42.0;
    s.load(empty);
    pdlpx::LpResult r = s.solve();
    CHECK(r.status == Status::Optimal && r.objective == 42.0);
    CHECK(!s.usedGpu());
    LpProblem bounds;  // min x, 1 <= x <= 4, no rows
    bounds.num_cols = 1;
    bounds.obj = {1.0};
    bounds.col_lower = {1.0};
    bounds.col_upper = {4.0};
    s.load(bounds);
    r = s.solve();
    std::vector<double> x = s.getPrimalValues();
    CHECK(r.status == Status::Optimal && x.size() == 1 && std::fabs(x[0] - 1.0) < 1e-12);
    CHECK(s.getBasis().empty());
    LpProblem unb;  // min -x, x >= 0, no rows
    unb.num_cols = 1;
    unb.obj = {-1.0};
    unb.col_lower = {0.0};
    unb.col_upper = {kInf};
    s.load(unb);
    CHECK(s.solve().status == Status::Unbounded);
    PdlpSolver moved(std::move(s));
    moved.load(empty);
    CHECK(moved.solve().status == Status::Optimal);
    return fails;
}

// The concurrent-root race of mipx (mip_solver.cpp:4470-4605): arms on their
// own threads and solvers share one stop flag, a std::atomic<bool> handed over
// through PdlpOptions::stop_flag exactly as the reference's race does; the first
// arm to finish sets it and the other returns IterLimit at its next check (or
// finishes first).
static int race() {
    LpProblem lp;  // a 300-row random-like LP: sum_j x_j <= 10 + i per row, max sum x
    lp.num_cols = 600;
    lp.num_rows = 300;
    lp.obj.assign(600, -1.0);
    lp.col_lower.assign(600, 0.0);
    lp.col_upper.assign(600, 5.0);
    lp.row_lower.assign(300, -kInf);
    lp.row_starts = {0};
    for (int i = 0; i < 300; ++i) {
        lp.row_upper.push_back(10.0 + i);
        for (int k = 0; k < 7; ++k) {
            lp.col_indices.push_back((i * 7 + k * 97) % 600);
            lp.values.push_back(1.0 + 0.1 * k);
        }
        std::vector<int32_t> row(lp.col_indices.end() - 7, lp.col_indices.end());
        std::vector<double> val(lp.values.end() - 7, lp.values.end());
        // columns sorted and distinct within the row
        std::vector<std::pair<int32_t, double>> e;
        for (int k = 0; k < 7; ++k) e.emplace_back(row[k], val[k]);
        std::sort(e.begin(), e.end());
        for (int k = 0; k < 7; ++k) {
            lp.col_indices[lp.col_indices.size() - 7 + k] = e[k].first;
            lp.values[lp.values.size() - 7 + k] = e[k].second;
        }
        lp.row_starts.push_back(static_cast<int32_t>(lp.values.size()));
    }
    std::atomic<bool> stop{false};
    pdlpx::LpResult res[2];
    std::atomic<int> first{-1};
    auto arm = [&](int k) {
        PdlpSolver s;
        pdlpx::PdlpOptions o;
        o.verbose = 0;
        o.max_iter = 200000;
        o.precision = k == 0 ? PDLPX_PREC_MIXED : PDLPX_PREC_FP64;
        o.primal_tol = o.dual_tol = o.optimality_tol = k == 0 ? 1e-4 : 1e-9;  // arm 1 needs far longer
        o.stop_flag = &stop;
        s.setOptions(o);
        s.load(lp);
        res[k] = s.solve();
        int expected = -1;
        if (first.compare_exchange_strong(expected, k)) stop.store(true);
    };
    std::thread a(arm, 0), b(arm, 1);
    a.join();
    b.join();
    const int w = first.load(), l = 1 - w;
    CHECK(res[w].status == Status::Optimal);
    CHECK(res[l].status == Status::IterLimit || res[l].status == Status::Optimal);
    std::printf("race: arm %d won, the other ended %d after %d iterations\n", w, static_cast<int>(res[l].status),
                res[l].iterations);
    return 0;
}

static int gpu() {
    PdlpSolver s;
    pdlpx::PdlpOptions o;
    o.verbose = 0;
    o.max_iter = 50000;
    s.setOptions(o);
    s.load(simpleLp());
    pdlpx::LpResult r = s.solve();
    CHECK(r.status == Status::Optimal && std::fabs(r.objective + 4.0) <= 1e-4);
    CHECK(s.usedGpu() && r.iterations > 0 && r.work_units > 0.0);
    CHECK(s.getStatus() == Status::Optimal && s.getObjective() == r.objective);
    CHECK(s.getPrimalValues().size() == 2 && s.getDualValues().size() == 1 && s.getReducedCosts().size() == 2);
    const std::vector<double> bad = {1.0};
    s.setWarmStart(bad, {});  // wrong sizes: ignored at solve time (pdlp.cpp:918-919)
    CHECK(s.solve().status == Status::Optimal);
    LpProblem mx = simpleLp();
    mx.sense = pdlpx::Sense::Maximize;
    mx.obj = {1.0, 1.0};
    s.load(mx);
    r = s.solve();
    CHECK(r.status == Status::Optimal && std::fabs(r.objective - 4.0) <= 1e-4);
    // x <= 1 as an appended row: max x + y stays 4 (y takes the rest)
    const std::vector<int32_t> starts = {0, 1}, idx = {0};
    const std::vector<double> vals = {1.0}, lo = {-kInf}, up = {1.0};
    s.addRows(starts, idx, vals, lo, up);
    r = s.solve();
    std::vector<double> x = s.getPrimalValues();
    CHECK(r.status == Status::Optimal && std::fabs(r.objective - 4.0) <= 1e-4 && x[0] <= 1.0 + 1e-4);
    s.setColBounds(1, 0.0, 2.0);  // y <= 2: max becomes 3
    r = s.solve();
    CHECK(r.status == Status::Optimal && std::fabs(r.objective - 3.0) <= 1e-4);
    // a flag raised before the solve stops it at the first check: IterLimit, as in the reference
    std::atomic<bool> raised{true};
    pdlpx::PdlpOptions so = o;
    so.stop_flag = &raised;
    s.setOptions(so);
    CHECK(s.solve().status == Status::IterLimit);
    s.setStopFlag(static_cast<const std::atomic<bool>*>(nullptr));  // cleared: solves again
    CHECK(s.solve().status == Status::Optimal);
    return race() + fails;
}

int main(int argc, char** argv) {
    if (argc > 1 && std::strcmp(argv[1], "gpu") == 0) return gpu() ? 1 : 0;
    return host() ? 1 : 0;
}
