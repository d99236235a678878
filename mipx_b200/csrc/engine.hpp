// Engine: one LP, its scaled copy, its device image and the solve loop.
// This is the C++ host side behind the C ABI (pdlpx.h); its public methods
// mirror mipx::PdlpSolver (include/mipx/pdlp.h:89-174).
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "pdlpx.h"
#include "problem.hpp"

namespace pdlpx {

struct DeviceLp;  // device buffers, graphs (engine.cu)

class Engine {
public:
    Engine();
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    void setOptions(const pdlpx_options& o) { opt_ = o; }
    const pdlpx_options& options() const { return opt_; }

    // Copies the problem (PdlpSolver::load, pdlp.cpp:445-455).  Returns PDLPX_*.
    int32_t load(int32_t m, int32_t n, int32_t nnz, const int32_t* rp, const int32_t* ci,
                 const double* v, const double* obj, const double* cl, const double* cu,
                 const double* rl, const double* ru, int32_t sense, double offset);
    int32_t solve(pdlpx_result* out);

    void setWarmStart(const double* x, int32_t nx, const double* y, int32_t ny);
    void clearWarmStart();
    void setStopFlag(const int32_t* f) { stop_flag_ = f; }
    void setStopCallback(pdlpx_stop_poll poll, void* ctx) {
        stop_poll_ = poll;
        stop_ctx_ = poll != nullptr ? ctx : nullptr;
    }
    bool stopRequested() const {
        return (stop_flag_ != nullptr && __atomic_load_n(stop_flag_, __ATOMIC_RELAXED) != 0) ||
               (stop_poll_ != nullptr && stop_poll_(stop_ctx_) != 0);
    }

    bool loaded() const { return loaded_; }
    int32_t status() const { return status_; }
    double objective() const { return objective_; }
    bool usedGpu() const { return used_gpu_; }
    const std::vector<double>& primal() const { return x_orig_; }
    const std::vector<double>& dual() const { return y_orig_; }
    void reducedCosts(std::vector<double>& rc) const;
    const HostLp& problem() const { return lp_; }
    const ScaledLp& scaled() const { return sc_; }

    // Incremental edits (pdlp.cpp:2833-2907): edit the original, rescale.
    void addRows(int32_t rows, const int32_t* starts, const int32_t* idx, const double* vals,
                 int32_t nvals, const double* lo, const double* up);
    void removeRows(const int32_t* rows, int32_t count);
    void setColBounds(int32_t col, double lo, double up);
    void setObjective(const double* obj, int32_t n);

    // Kernel timing for the roofline report (pdlpx_time_kernels): precision
    // PDLPX_PREC_MIXED / PDLPX_PREC_FP64 / -1 (the last solve's final one).
    int32_t timeKernels(int32_t precision, int32_t reps, int64_t flush_bytes, double* ms_primal, double* ms_dual,
                        double* ms_check);
    // Step-kernel times sampled inside the last solve (pdlpx_get_step_times).
    void stepTimes(int32_t precision, double* ms_primal, double* ms_dual, int32_t* samples) const {
        const int p = precision == PDLPX_PREC_FP64 ? 1 : 0;
        const int k = step_samples_[p];
        if (ms_primal) *ms_primal = k > 0 ? step_ms_[p][0] / k : 0.0;
        if (ms_dual) *ms_dual = k > 0 ? step_ms_[p][1] / k : 0.0;
        if (samples) *samples = k;
    }
    int32_t launchConfig(int32_t* ga, int32_t* gat, int32_t* bp, int32_t* bd) const;
    int32_t hotPrefix(int32_t precision, int32_t* primal, int32_t* dual) const;
    int32_t longTiles(int32_t* chunks, int32_t* groups) const;

    std::string last_error;

private:
    void rescale();
    int32_t solveTrivial(pdlpx_result* out);
    int32_t solveDevice(pdlpx_result* out);

    pdlpx_options opt_{};
    HostLp lp_;
    ScaledLp sc_;
    bool loaded_ = false;
    std::vector<double> warm_x_, warm_y_;
    bool has_warm_ = false;
    const int32_t* stop_flag_ = nullptr;
    pdlpx_stop_poll stop_poll_ = nullptr;
    void* stop_ctx_ = nullptr;

    int32_t status_ = PDLPX_STATUS_ERROR;
    double objective_ = 0.0;
    int32_t iterations_ = 0;
    bool used_gpu_ = false;
    std::vector<double> x_orig_, y_orig_;
    double step_ms_[2][2] = {{0, 0}, {0, 0}};  // [FP32 / FP64 kernels][primal / dual] sums of the last solve
    int step_samples_[2] = {0, 0};

    std::unique_ptr<DeviceLp> dev_;
};

// Threads per row for the CSR kernels, from the mean row length.
int32_t pickGroup(int64_t nnz, int32_t rows);

// Batched solve of independent LPs packed into one device image (batch.cu).
int32_t batchSolve(int32_t count, const pdlpx_lp* lps, const pdlpx_options& o, pdlpx_result* results,
                   double* const* x_out, double* const* y_out, std::string& err);

// Independent LPs over several devices (batch.cu): deterministic
// longest-processing-time sharding, and the batch solved per device.
void shardLps(int32_t count, const int64_t* weights, int32_t ndev, int32_t* device_of);
int32_t batchSolveDevices(int32_t count, const pdlpx_lp* lps, const pdlpx_options& o, const int32_t* devices,
                          int32_t ndev, pdlpx_result* results, double* const* x_out, double* const* y_out,
                          std::string& err);

// The persistent batch cycle's grid barrier run on its own (batch.cu).
int32_t gridBarrierCheck(int32_t device, int32_t blocks, int32_t rounds, int32_t stall, int32_t* barrier_error,
                         double* seconds, std::string& err);

// Message returned by pdlpx_last_error(NULL) on this thread (calls without a handle).
void setGlobalError(const std::string& msg);

// Device SpMV used by pdlpx_csr_spmv (host buffers in/out).
int32_t deviceSpmv(int32_t rows, int32_t cols, int32_t nnz, const int32_t* rp, const int32_t* ci,
                   const double* val, const double* x, double* y, int32_t precision, int32_t group,
                   std::string& err);

}  // namespace pdlpx
