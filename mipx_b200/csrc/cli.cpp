// pdlpx_cli: command-line LP solve with mipx's `--pdlp` front end and output.
//
//   pdlpx_cli model.mps[.gz] [--pdlp] [--quiet | --verbose] [--print-backend]
//             [--time-limit S] [--pdlp-opt-norm l2|linf] [--tol T] [--fp64]
//             [--threads N] [--gpu | --no-gpu] [--gpu-min-rows N] [--gpu-min-nnz N]
//             [--no-presolve] [--relax-integrality]
//
// It reads the MPS file with the library's reader (pdlpx_read_mps), solves the
// LP relaxation (integrality marks are ignored) through the C++ mirror of
// PdlpSolver, and prints the lines mipx's CLI prints for an LP solve
// (src/cli/main.cpp:553-607): the status line, "PDLP backend: GPU" with
// --print-backend or --verbose, then the stable summary lines that benchmark
// scripts parse -- "Status: ...", "Objective: %.10e", "Iterations: %d",
// "Work units: %.2f", "Time: %.2fs".  Flags mipx accepts for other solvers or
// for its presolve (--threads, --no-presolve, --relax-integrality, the GPU
// thresholds) are accepted and have no effect: every solve runs on the GPU and
// there is no presolve.  Exit status 0 after a solve (any LP status), 1 on a
// usage or read error.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pdlpx.hpp"

namespace {

const char* statusText(pdlpx::Status s) {
    switch (s) {
        case pdlpx::Status::Optimal:
            return "Optimal";
        case pdlpx::Status::Infeasible:
            return "Infeasible";
        case pdlpx::Status::Unbounded:
            return "Unbounded";
        case pdlpx::Status::IterLimit:
            return "Iteration limit";
        case pdlpx::Status::TimeLimit:
            return "Time limit";
        default:
            return "Error";
    }
}

int usage() {
    std::fprintf(stderr,
                 "usage: pdlpx_cli model.mps[.gz] [--pdlp] [--quiet|--verbose] [--print-backend]\n"
                 "                 [--time-limit S] [--pdlp-opt-norm l2|linf] [--tol T] [--fp64]\n");
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    std::string path;
    bool quiet = false, verbose = false, print_backend = false, fp64 = false;
    double time_limit = -1.0, tol = -1.0;
    int norm = PDLPX_NORM_L2;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto value = [&]() -> const char* { return i + 1 < argc ? argv[++i] : nullptr; };
        if (a == "--quiet") {
            quiet = true;
        } else if (a == "--verbose") {
            verbose = true;
        } else if (a == "--print-backend") {
            print_backend = true;
        } else if (a == "--fp64") {
            fp64 = true;
        } else if (a == "--time-limit" || a == "--time_limit") {
            const char* v = value();
            if (!v) return usage();
            time_limit = std::atof(v);
        } else if (a == "--tol") {
            const char* v = value();
            if (!v) return usage();
            tol = std::atof(v);
        } else if (a == "--pdlp-opt-norm") {
            const char* v = value();
            if (!v) return usage();
            norm = std::strcmp(v, "linf") == 0 || std::strcmp(v, "inf") == 0 ? PDLPX_NORM_LINF : PDLPX_NORM_L2;
        } else if (a == "--threads" || a == "--gpu-min-rows" || a == "--gpu-min-nnz") {
            if (!value()) return usage();
        } else if (a == "--pdlp" || a == "--gpu" || a == "--no-gpu" || a == "--no-presolve" ||
                   a == "--relax-integrality") {
            // accepted for command-line compatibility
        } else if (!a.empty() && a[0] == '-') {
            std::fprintf(stderr, "unknown option %s\n", a.c_str());
            return usage();
        } else {
            path = a;
        }
    }
    if (path.empty()) return usage();

    pdlpx_gen_lp g{};
    if (pdlpx_read_mps(path.c_str(), &g) != PDLPX_OK) {
        std::fprintf(stderr, "Error: %s\n", pdlpx_last_error(nullptr));
        return 1;
    }
    pdlpx::LpProblem lp;
    lp.num_rows = g.m;
    lp.num_cols = g.n;
    lp.obj.assign(g.obj, g.obj + g.n);
    lp.col_lower.assign(g.col_lb, g.col_lb + g.n);
    lp.col_upper.assign(g.col_ub, g.col_ub + g.n);
    lp.row_lower.assign(g.row_lb, g.row_lb + g.m);
    lp.row_upper.assign(g.row_ub, g.row_ub + g.m);
    lp.row_starts.assign(g.row_ptr, g.row_ptr + g.m + 1);
    lp.col_indices.assign(g.col_idx, g.col_idx + g.nnz);
    lp.values.assign(g.val, g.val + g.nnz);
    lp.obj_offset = g.obj_offset;
    pdlpx_free_lp(&g);
    if (!quiet) std::printf("LP %s: %d rows, %d columns, %zu nonzeros\n", path.c_str(), lp.num_rows, lp.num_cols,
                            lp.values.size());

    pdlpx::PdlpOptions o;
    o.verbose = verbose ? 1 : 0;
    o.max_solve_seconds = time_limit;
    o.optimality_norm = norm;
    if (tol > 0.0) o.primal_tol = o.dual_tol = o.optimality_tol = tol;
    if (fp64) o.precision = PDLPX_PREC_FP64;
    pdlpx::PdlpSolver s;
    s.setOptions(o);
    s.load(lp);
    const auto t0 = std::chrono::steady_clock::now();
    const pdlpx::LpResult r = s.solve();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (verbose || print_backend) std::printf("PDLP backend: %s\n", s.usedGpu() ? "GPU" : "CPU");
    std::fflush(stdout);
    std::printf("\n");
    if (r.status == pdlpx::Status::Optimal)
        std::printf("Optimal: %.10e (%d iterations)\n", r.objective, r.iterations);
    else
        std::printf("Status: %s\n", statusText(r.status));
    if (r.status == pdlpx::Status::Error) std::printf("Error detail: %s\n", s.lastError());
    std::printf("Status: %s\n", statusText(r.status));
    std::printf("Objective: %.10e\n", r.objective);
    std::printf("Iterations: %d\n", r.iterations);
    std::printf("Work units: %.2f\n", r.work_units);
    std::printf("Time: %.2fs\n", secs);
    return 0;
}
