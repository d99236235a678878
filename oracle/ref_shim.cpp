// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// extern "C" shim over the reference's own mipx::PdlpSolver.  oracle/Makefile
// compiles this file together with the reference's sources where they lie
// (src/lp/pdlp.cpp, src/lp/sparse_matrix.cpp of spoorendonk/mipx) into
// oracle/_ref/libmipx_pdlp_ref.so (CPU build) and, with MIPX_HAS_CUDA, into
// oracle/_ref/libmipx_pdlp_ref_gpu.so (the reference's cuSPARSE FP64 GPU path).
// The tests use it to pin the oracle restatement (oracle/pdlp_oracle.cpp) and
// bench.py uses the CPU build as the reference arm.
#include <atomic>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

#include "mipx/pdlp.h"
#include "pdlpx.h"

namespace {

mipx::PdlpOptions toRefOptions(const pdlpx_options& o) {
    mipx::PdlpOptions r;
    r.max_iter = o.max_iter;
    r.optimality_tol = o.optimality_tol;
    r.primal_tol = o.primal_tol;
    r.dual_tol = o.dual_tol;
    r.max_solve_seconds = o.max_solve_seconds;
    r.optimality_norm = o.optimality_norm == PDLPX_NORM_LINF ? mipx::PdlpOptimalityNorm::LInf
                                                             : mipx::PdlpOptimalityNorm::L2;
    r.sv_max_iter = o.sv_max_iter;
    r.sv_tol = o.sv_tol;
    r.adaptive_step = o.adaptive_step != 0;
    r.adaptive_step_down = o.adaptive_step_down;
    r.adaptive_step_up = o.adaptive_step_up;
    r.adaptive_step_min = o.adaptive_step_min;
    r.adaptive_step_max = o.adaptive_step_max;
    r.primal_weight = o.primal_weight;
    r.update_primal_weight = o.update_primal_weight != 0;
    r.pid_kp = o.pid_kp;
    r.pid_ki = o.pid_ki;
    r.pid_kd = o.pid_kd;
    r.pid_i_smooth = o.pid_i_smooth;
    r.restart_sufficient_decay = o.restart_sufficient_decay;
    r.restart_necessary_decay = o.restart_necessary_decay;
    r.restart_artificial_fraction = o.restart_artificial_fraction;
    r.termination_eval_frequency = o.termination_eval_frequency;
    r.matrix_zero_tol = o.matrix_zero_tol;
    r.enable_polishing = o.enable_polishing != 0;
    r.polish_primal_tol = o.polish_primal_tol;
    r.polish_dual_tol = o.polish_dual_tol;
    r.polish_max_iter = o.polish_max_iter;
    r.do_ruiz_scaling = o.do_ruiz_scaling != 0;
    r.ruiz_iterations = o.ruiz_iterations;
    r.do_pock_chambolle_scaling = o.do_pock_chambolle_scaling != 0;
    r.do_bound_obj_rescaling = o.do_bound_obj_rescaling != 0;
    r.preconditioner_refresh = o.preconditioner_refresh != 0;
    r.preconditioner_refresh_ratio = o.preconditioner_refresh_ratio;
    r.anderson_acceleration = o.anderson_acceleration != 0;
    r.anderson_window_size = o.anderson_window_size;
    r.anderson_regularization = o.anderson_regularization;
    r.use_gpu = o.use_gpu != 0;
    r.gpu_min_rows = o.gpu_min_rows;
    r.gpu_min_nnz = o.gpu_min_nnz;
    r.verbose = o.verbose != 0;
    return r;
}

mipx::LpProblem toRefProblem(const pdlpx_lp& lp) {
    mipx::LpProblem p;
    p.sense = lp.sense == PDLPX_MAXIMIZE ? mipx::Sense::Maximize : mipx::Sense::Minimize;
    p.num_cols = lp.n;
    p.num_rows = lp.m;
    p.obj.assign(lp.obj, lp.obj + lp.n);
    p.col_lower.assign(lp.col_lb, lp.col_lb + lp.n);
    p.col_upper.assign(lp.col_ub, lp.col_ub + lp.n);
    p.col_type.assign(static_cast<size_t>(lp.n), mipx::VarType::Continuous);
    p.row_lower.assign(lp.row_lb, lp.row_lb + lp.m);
    p.row_upper.assign(lp.row_ub, lp.row_ub + lp.m);
    std::vector<mipx::Triplet> trips;
    trips.reserve(static_cast<size_t>(lp.nnz));
    for (int i = 0; i < lp.m; ++i)
        for (int k = lp.row_ptr[i]; k < lp.row_ptr[i + 1]; ++k)
            trips.push_back({i, lp.col_idx[k], lp.val[k]});
    p.matrix = mipx::SparseMatrix(lp.m, lp.n, std::move(trips));
    p.obj_offset = lp.obj_offset;
    return p;
}

}  // namespace

extern "C" {

// Solve one LP with the reference PdlpSolver.  Returns 0; fills res, x[n], y[m]
// (x / y may be NULL).  stop_flag may be NULL.
int ref_pdlp_solve(const pdlpx_lp* lp, const pdlpx_options* opts, pdlpx_result* res, double* x,
                   double* y) {
    if (lp == nullptr || opts == nullptr || res == nullptr) return PDLPX_E_INVALID;
    mipx::PdlpSolver solver;
    solver.setOptions(toRefOptions(*opts));
    solver.load(toRefProblem(*lp));
    if (lp->warm_x != nullptr && lp->warm_y != nullptr) {
        solver.setWarmStart(std::span<const double>(lp->warm_x, static_cast<size_t>(lp->n)),
                            std::span<const double>(lp->warm_y, static_cast<size_t>(lp->m)));
    }
    auto t0 = std::chrono::steady_clock::now();
    mipx::LpResult r = solver.solve();
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::memset(res, 0, sizeof(*res));
    res->status = static_cast<int32_t>(r.status);
    res->objective = r.objective;
    res->iterations = r.iterations;
    res->work_units = r.work_units;
    res->solve_seconds = secs;
    res->used_gpu = solver.usedGpu() ? 1 : 0;
    if (x != nullptr) {
        auto v = solver.getPrimalValues();
        for (size_t j = 0; j < v.size() && j < static_cast<size_t>(lp->n); ++j) x[j] = v[j];
    }
    if (y != nullptr) {
        auto v = solver.getDualValues();
        for (size_t i = 0; i < v.size() && i < static_cast<size_t>(lp->m); ++i) y[i] = v[i];
    }
    return PDLPX_OK;
}

// Reduced costs c + A^T y of the last solve are not kept across calls; this
// variant solves and returns them (rc[n]).
int ref_pdlp_solve_rc(const pdlpx_lp* lp, const pdlpx_options* opts, pdlpx_result* res,
                      double* rc) {
    mipx::PdlpSolver solver;
    solver.setOptions(toRefOptions(*opts));
    solver.load(toRefProblem(*lp));
    mipx::LpResult r = solver.solve();
    res->status = static_cast<int32_t>(r.status);
    res->objective = r.objective;
    res->iterations = r.iterations;
    res->work_units = r.work_units;
    auto v = solver.getReducedCosts();
    for (size_t j = 0; j < v.size(); ++j) rc[j] = v[j];
    return PDLPX_OK;
}

// A reference solver kept across calls, for the CPU baseline timing: open
// copies and loads the LP once (the reference's load runs its scaling
// pipeline); every run then calls the reference's solve() with a new iteration
// cap and power-iteration cap and reports its wall time in res->solve_seconds.
struct RefHandle {
    mipx::PdlpSolver solver;
    mipx::PdlpOptions opts;
};

void* ref_pdlp_open(const pdlpx_lp* lp, const pdlpx_options* opts) {
    if (lp == nullptr || opts == nullptr) return nullptr;
    auto* h = new RefHandle();
    h->opts = toRefOptions(*opts);
    h->solver.setOptions(h->opts);
    h->solver.load(toRefProblem(*lp));
    return h;
}

int ref_pdlp_run(void* handle, int32_t max_iter, int32_t sv_max_iter, pdlpx_result* res) {
    auto* h = static_cast<RefHandle*>(handle);
    if (h == nullptr || res == nullptr) return PDLPX_E_INVALID;
    h->opts.max_iter = max_iter;
    h->opts.sv_max_iter = sv_max_iter;
    h->solver.setOptions(h->opts);
    auto t0 = std::chrono::steady_clock::now();
    mipx::LpResult r = h->solver.solve();
    std::memset(res, 0, sizeof(*res));
    res->solve_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    res->status = static_cast<int32_t>(r.status);
    res->objective = r.objective;
    res->iterations = r.iterations;
    res->work_units = r.work_units;
    res->used_gpu = h->solver.usedGpu() ? 1 : 0;
    return PDLPX_OK;
}

void ref_pdlp_close(void* handle) { delete static_cast<RefHandle*>(handle); }

// The concurrent-root race pattern of mipx (mip_solver.cpp:4470-4605) over the
// reference's own PdlpSolver class: two arms on their own threads, each with
// its own solver and options, share one std::atomic<bool> through
// PdlpOptions::stop_flag; the first arm to finish raises it and the other ends
// at its next check with IterLimit (or finishes first).  winner = 0 or 1.
int ref_pdlp_race(const pdlpx_lp* lp, const pdlpx_options* arm0, const pdlpx_options* arm1, pdlpx_result* r0,
                  pdlpx_result* r1, int* winner) {
    if (lp == nullptr || arm0 == nullptr || arm1 == nullptr || r0 == nullptr || r1 == nullptr || winner == nullptr)
        return PDLPX_E_INVALID;
    const mipx::LpProblem problem = toRefProblem(*lp);
    std::atomic<bool> stop{false};
    std::atomic<int> first{-1};
    pdlpx_result* out[2] = {r0, r1};
    const pdlpx_options* opts[2] = {arm0, arm1};
    auto arm = [&](int k) {
        mipx::PdlpSolver solver;
        mipx::PdlpOptions o = toRefOptions(*opts[k]);
        o.stop_flag = &stop;
        solver.setOptions(o);
        solver.load(problem);
        const mipx::LpResult r = solver.solve();
        int expected = -1;
        if (first.compare_exchange_strong(expected, k)) stop.store(true);
        std::memset(out[k], 0, sizeof(pdlpx_result));
        out[k]->status = static_cast<int32_t>(r.status);
        out[k]->objective = r.objective;
        out[k]->iterations = r.iterations;
        out[k]->work_units = r.work_units;
        out[k]->used_gpu = solver.usedGpu() ? 1 : 0;
    };
    std::thread a(arm, 0), b(arm, 1);
    a.join();
    b.join();
    *winner = first.load();
    return PDLPX_OK;
}

int ref_has_cuda(void) {
#ifdef MIPX_HAS_CUDA
    return 1;
#else
    return 0;
#endif
}

}  // extern "C"
