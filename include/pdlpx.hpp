/* C++ mirror of mipx's PDLP solver interface over the pdlpx C ABI.
 *
 * The types and methods follow the reference's public interface name for name
 * (class PdlpSolver : LpSolver, include/mipx/pdlp.h:89-174 and
 * include/mipx/lp_solver.h:11-60; PdlpOptions, pdlp.h:19-87; Status,
 * include/mipx/core.h:11-19; LpProblem's CSR layout, include/mipx/lp_problem.h:14-64)
 * with the reference's behaviour at the boundary: load() copies the problem,
 * getters return vectors by value in original space, nothing throws, a failed
 * call leaves Status::Error, a warm start of the wrong size is ignored, and
 * getBasis() / setBasis() are empty (PDLP has no basis).  Header only; link
 * with -lpdlpx.
 *
 *   pdlpx::LpProblem lp;  ... fill the CSR rows, bounds, objective ...
 *   pdlpx::PdlpSolver s;
 *   pdlpx::PdlpOptions o;  o.verbose = 0;  s.setOptions(o);
 *   s.load(lp);
 *   pdlpx::LpResult r = s.solve();           // r.status, r.objective, r.iterations, r.work_units
 *   std::vector<double> x = s.getPrimalValues();
 */
#pragma once

#include <atomic>
#include <cstdint>
#include <limits>
#include <span>
#include <utility>
#include <vector>

#include "pdlpx.h"

namespace pdlpx {

using Real = double;
using Index = int32_t;
using Int = int32_t;
inline constexpr Real kInf = std::numeric_limits<Real>::infinity();

/* Same numbering as mipx::Status (core.h:11-19) and PDLPX_STATUS_*. */
enum class Status : int32_t { Optimal = 0, Infeasible, Unbounded, IterLimit, TimeLimit, NodeLimit, Error };
enum class Sense : int32_t { Minimize = PDLPX_MINIMIZE, Maximize = PDLPX_MAXIMIZE };
enum class BasisStatus { Basic, AtLower, AtUpper, Fixed, Free };

struct LpResult {
    Status status = Status::Error;
    Real objective = 0.0;
    Int iterations = 0;
    double work_units = 0.0;
};

/* The reference's PdlpOptions fields under the same names and defaults
 * (booleans are int32 0/1), plus the engine's launch and batching knobs.
 * stop_flag has the reference's type (pdlp.h:86): code that sets
 * `opts.stop_flag = &flag; solver.setOptions(opts);` compiles unchanged, and
 * the solver polls the atomic once per restart cycle through the C ABI's stop
 * callback (no mirroring thread). */
struct PdlpOptions : pdlpx_options {
    PdlpOptions() { pdlpx_options_default(this); }
    const std::atomic<bool>* stop_flag = nullptr;
};

/* An LP in the reference's ranged form: row_lower <= A x <= row_upper,
 * col_lower <= x <= col_upper, A as CSR rows (row_starts has num_rows + 1 entries). */
struct LpProblem {
    Sense sense = Sense::Minimize;
    Index num_cols = 0, num_rows = 0;
    std::vector<Real> obj, col_lower, col_upper, row_lower, row_upper;
    Real obj_offset = 0.0;
    std::vector<Index> row_starts{0}, col_indices;
    std::vector<Real> values;
};

class PdlpSolver {
public:
    PdlpSolver() {
        if (pdlpx_create(&options_, &h_) != PDLPX_OK) h_ = nullptr;
    }
    ~PdlpSolver() {
        if (h_) pdlpx_destroy(h_);
    }
    PdlpSolver(const PdlpSolver&) = delete;
    PdlpSolver& operator=(const PdlpSolver&) = delete;
    PdlpSolver(PdlpSolver&& o) noexcept { swap(o); }
    PdlpSolver& operator=(PdlpSolver&& o) noexcept {
        swap(o);
        return *this;
    }

    /* Copies the problem (pdlp.cpp:445-455); clears any warm start. */
    void load(const LpProblem& p) {
        status_ = Status::Error;
        objective_ = 0.0;
        if (!h_) return;
        const int32_t nnz = static_cast<int32_t>(p.values.size());
        if (pdlpx_load_csr(h_, p.num_rows, p.num_cols, nnz, p.row_starts.data(), p.col_indices.data(),
                           p.values.data(), p.obj.data(), p.col_lower.data(), p.col_upper.data(),
                           p.row_lower.data(), p.row_upper.data(), static_cast<int32_t>(p.sense),
                           p.obj_offset) != PDLPX_OK)
            return;
        pdlpx_clear_warm_start(h_);
    }

    /* Solves on the GPU; a call that fails reports Status::Error (pdlp.cpp:1979-1983). */
    LpResult solve() {
        LpResult out;
        pdlpx_result r{};
        if (!h_ || pdlpx_solve(h_, &r) != PDLPX_OK) {
            status_ = Status::Error;
            objective_ = 0.0;
            return out;
        }
        status_ = static_cast<Status>(r.status);
        objective_ = r.objective;
        out.status = status_;
        out.objective = r.objective;
        out.iterations = r.iterations;
        out.work_units = r.work_units;
        return out;
    }

    Status getStatus() const { return status_; }
    Real getObjective() const { return objective_; }

    std::vector<Real> getPrimalValues() const {
        std::vector<Real> x(static_cast<size_t>(dims().second));
        if (h_ && !x.empty()) pdlpx_get_primal(h_, x.data(), static_cast<int32_t>(x.size()));
        return x;
    }
    std::vector<Real> getDualValues() const {
        std::vector<Real> y(static_cast<size_t>(dims().first));
        if (h_ && !y.empty()) pdlpx_get_dual(h_, y.data(), static_cast<int32_t>(y.size()));
        return y;
    }
    std::vector<Real> getReducedCosts() const {
        std::vector<Real> rc(static_cast<size_t>(dims().second));
        if (h_ && !rc.empty()) pdlpx_get_reduced_costs(h_, rc.data(), static_cast<int32_t>(rc.size()));
        return rc;
    }

    std::vector<BasisStatus> getBasis() const { return {}; }
    void setBasis(std::span<const BasisStatus>) {}

    /* Incremental edits (pdlp.cpp:2833-2907); invalid input is ignored, as there. */
    void addRows(std::span<const Index> starts, std::span<const Index> indices, std::span<const Real> values,
                 std::span<const Real> lower, std::span<const Real> upper) {
        if (!h_ || starts.empty() || lower.size() + 1 != starts.size() || upper.size() != lower.size()) return;
        pdlpx_add_rows(h_, static_cast<int32_t>(lower.size()), starts.data(), indices.data(), values.data(),
                       static_cast<int32_t>(values.size()), lower.data(), upper.data());
    }
    void removeRows(std::span<const Index> rows) {
        if (h_) pdlpx_remove_rows(h_, rows.data(), static_cast<int32_t>(rows.size()));
    }
    void setColBounds(Index col, Real lower, Real upper) {
        if (h_) pdlpx_set_col_bounds(h_, col, lower, upper);
    }
    void setObjective(std::span<const Real> obj) {
        if (h_) pdlpx_set_objective(h_, obj.data(), static_cast<int32_t>(obj.size()));
    }

    /* Warm start in original space; ignored at solve time when the sizes do not match. */
    void setWarmStart(std::span<const Real> x, std::span<const Real> y) {
        if (h_)
            pdlpx_set_warm_start(h_, x.data(), static_cast<int32_t>(x.size()), y.data(),
                                 static_cast<int32_t>(y.size()));
    }
    void clearWarmStart() {
        if (h_) pdlpx_clear_warm_start(h_);
    }

    void setOptions(const PdlpOptions& options) {
        options_ = options;
        if (h_) pdlpx_set_options(h_, &options_);
        applyStopFlag();
    }
    const PdlpOptions& options() const { return options_; }
    bool usedGpu() const {
        int32_t u = 0;
        if (h_) pdlpx_used_gpu(h_, &u);
        return u != 0;
    }

    /* Cancellation (PdlpOptions::stop_flag of the reference, pdlp.h:86): polled
     * once per restart cycle; true ends the solve with Status::IterLimit. */
    void setStopFlag(const std::atomic<bool>* flag) {
        options_.stop_flag = flag;
        applyStopFlag();
    }
    /* The same with a plain int32 flag (read with an atomic load). */
    void setStopFlag(const int32_t* flag) {
        if (h_) pdlpx_set_stop_flag(h_, flag);
    }
    const char* lastError() const { return h_ ? pdlpx_last_error(h_) : "solver handle not created"; }

private:
    static int32_t pollAtomic(void* ctx) {
        return static_cast<const std::atomic<bool>*>(ctx)->load(std::memory_order_relaxed) ? 1 : 0;
    }
    void applyStopFlag() {
        if (!h_) return;
        const std::atomic<bool>* f = options_.stop_flag;
        pdlpx_set_stop_callback(h_, f != nullptr ? &PdlpSolver::pollAtomic : nullptr,
                                const_cast<void*>(static_cast<const void*>(f)));
    }
    std::pair<int32_t, int32_t> dims() const {
        int32_t m = 0, n = 0, z = 0;
        if (h_) pdlpx_get_dims(h_, &m, &n, &z);
        return {m, n};
    }
    void swap(PdlpSolver& o) noexcept {
        std::swap(h_, o.h_);
        std::swap(options_, o.options_);
        std::swap(status_, o.status_);
        std::swap(objective_, o.objective_);
    }

    pdlpx_solver* h_ = nullptr;
    PdlpOptions options_{};
    Status status_ = Status::Error;
    Real objective_ = 0.0;
};

}  // namespace pdlpx
