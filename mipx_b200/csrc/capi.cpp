// C ABI of the engine (include/pdlpx.h).  Thin: argument checks, exception
// barrier, delegation to pdlpx::Engine.  No call throws across the boundary.
#include <cmath>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "engine.hpp"
#include "pdlpx.h"

struct pdlpx_solver {
    pdlpx::Engine engine;
};

namespace {

thread_local std::string g_last_error;

}  // namespace

void pdlpx::setGlobalError(const std::string& msg) { g_last_error = msg; }

namespace {

template <class F>
int32_t guarded(pdlpx_solver* h, F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        if (h) h->engine.last_error = "host allocation failed";
        return PDLPX_E_NOMEM;
    } catch (const std::exception& e) {
        if (h) h->engine.last_error = e.what();
        return PDLPX_E_INVALID;
    } catch (...) {
        if (h) h->engine.last_error = "unknown exception";
        return PDLPX_E_INVALID;
    }
}

}  // namespace

extern "C" {

void pdlpx_options_default(pdlpx_options* o) {
    if (o == nullptr) return;
    std::memset(o, 0, sizeof(*o));
    o->max_iter = 4000000;
    o->optimality_tol = 5e-5;
    o->primal_tol = 5e-5;
    o->dual_tol = 5e-5;
    o->max_solve_seconds = -1.0;
    o->optimality_norm = PDLPX_NORM_L2;
    o->sv_max_iter = 5000;
    o->sv_tol = 1e-4;
    o->adaptive_step = 0;
    o->adaptive_step_down = 0.7;
    o->adaptive_step_up = 1.0;
    o->adaptive_step_min = 1e-6;
    o->adaptive_step_max = 1e3;
    o->primal_weight = 1.0;
    o->update_primal_weight = 1;
    o->pid_kp = 0.99;
    o->pid_ki = 0.01;
    o->pid_kd = 0.0;
    o->pid_i_smooth = 0.3;
    o->restart_sufficient_decay = 0.2;
    o->restart_necessary_decay = 0.5;
    o->restart_artificial_fraction = 0.36;
    o->termination_eval_frequency = 200;
    o->matrix_zero_tol = 0.0;
    o->enable_polishing = 1;
    o->polish_primal_tol = 1e-6;
    o->polish_dual_tol = 1e-6;
    o->polish_max_iter = 500000;
    o->do_ruiz_scaling = 1;
    o->ruiz_iterations = 10;
    o->do_pock_chambolle_scaling = 1;
    o->do_bound_obj_rescaling = 1;
    o->preconditioner_refresh = 0;
    o->preconditioner_refresh_ratio = 10.0;
    o->anderson_acceleration = 0;
    o->anderson_window_size = 5;
    o->anderson_regularization = 1e-10;
    o->use_gpu = 1;
    o->gpu_min_rows = 512;
    o->gpu_min_nnz = 10000;
    o->verbose = 1;
    o->precision = PDLPX_PREC_MIXED;
    o->device = 0;
    o->fp64_switch = 1;
    o->spmv_group_a = 0;
    o->spmv_group_at = 0;
    o->autotune = 0;
    o->shape_primal = 0;
    o->shape_dual = 0;
    o->batch_pack_mb = 0;
    o->batch_compact = 1;
    o->batch_sell = 1;
    o->scale_on_device = -1;
    o->sell = -1;
    o->reference_fixed_columns = 0;
    o->hot_cache = 0;
    o->long_tiles = -1;
    o->batch_persistent = 0;
    o->sell_window = 0;
}

const char* pdlpx_error_string(int32_t code) {
    switch (code) {
        case PDLPX_OK: return "ok";
        case PDLPX_E_INVALID: return "invalid argument";
        case PDLPX_E_NOT_LOADED: return "no problem loaded";
        case PDLPX_E_CUDA: return "CUDA error";
        case PDLPX_E_NOMEM: return "out of memory";
        case PDLPX_E_NO_DEVICE: return "no CUDA device";
        case PDLPX_E_TIMEOUT: return "device wait timed out";
        case PDLPX_E_BUSY: return "busy";
        case PDLPX_E_UNKNOWN_TICKET: return "unknown ticket";
        default: return "unknown error";
    }
}

const char* pdlpx_last_error(const pdlpx_solver* h) {
    if (h == nullptr) return g_last_error.c_str();
    return h->engine.last_error.c_str();
}

int32_t pdlpx_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

const char* pdlpx_version(void) { return "pdlpx 0.1 (sm_100a)"; }

void pdlpx_struct_sizes(int32_t* sizes) {
    if (sizes == nullptr) return;
    sizes[0] = static_cast<int32_t>(sizeof(pdlpx_options));
    sizes[1] = static_cast<int32_t>(sizeof(pdlpx_result));
    sizes[2] = static_cast<int32_t>(sizeof(pdlpx_lp));
    sizes[3] = static_cast<int32_t>(sizeof(pdlpx_gen_lp));
    sizes[4] = static_cast<int32_t>(sizeof(pdlpx_server_config));
    sizes[5] = static_cast<int32_t>(sizeof(pdlpx_server_stats));
}

int32_t pdlpx_create(const pdlpx_options* opts, pdlpx_solver** out) {
    if (out == nullptr) return PDLPX_E_INVALID;
    *out = nullptr;
    auto* h = new (std::nothrow) pdlpx_solver();
    if (h == nullptr) return PDLPX_E_NOMEM;
    if (opts != nullptr) h->engine.setOptions(*opts);
    *out = h;
    return PDLPX_OK;
}

int32_t pdlpx_destroy(pdlpx_solver* h) {
    delete h;
    return PDLPX_OK;
}

int32_t pdlpx_set_options(pdlpx_solver* h, const pdlpx_options* opts) {
    if (h == nullptr || opts == nullptr) return PDLPX_E_INVALID;
    h->engine.setOptions(*opts);
    return PDLPX_OK;
}

int32_t pdlpx_get_options(const pdlpx_solver* h, pdlpx_options* out) {
    if (h == nullptr || out == nullptr) return PDLPX_E_INVALID;
    *out = h->engine.options();
    return PDLPX_OK;
}

int32_t pdlpx_load_csr(pdlpx_solver* h, int32_t m, int32_t n, int32_t nnz, const int32_t* row_ptr,
                       const int32_t* col_idx, const double* val, const double* obj, const double* col_lb,
                       const double* col_ub, const double* row_lb, const double* row_ub, int32_t sense,
                       double obj_offset) {
    if (h == nullptr) return PDLPX_E_INVALID;
    return guarded(h, [&] {
        return h->engine.load(m, n, nnz, row_ptr, col_idx, val, obj, col_lb, col_ub, row_lb, row_ub, sense,
                              obj_offset);
    });
}

int32_t pdlpx_set_warm_start(pdlpx_solver* h, const double* x, int32_t nx, const double* y, int32_t ny) {
    if (h == nullptr || (nx > 0 && x == nullptr) || (ny > 0 && y == nullptr) || nx < 0 || ny < 0)
        return PDLPX_E_INVALID;
    return guarded(h, [&] {
        h->engine.setWarmStart(x, nx, y, ny);
        return PDLPX_OK;
    });
}

int32_t pdlpx_clear_warm_start(pdlpx_solver* h) {
    if (h == nullptr) return PDLPX_E_INVALID;
    h->engine.clearWarmStart();
    return PDLPX_OK;
}

int32_t pdlpx_set_stop_flag(pdlpx_solver* h, const int32_t* flag) {
    if (h == nullptr) return PDLPX_E_INVALID;
    h->engine.setStopFlag(flag);
    return PDLPX_OK;
}

int32_t pdlpx_set_stop_callback(pdlpx_solver* h, pdlpx_stop_poll poll, void* ctx) {
    if (h == nullptr) return PDLPX_E_INVALID;
    h->engine.setStopCallback(poll, ctx);
    return PDLPX_OK;
}

int32_t pdlpx_solve(pdlpx_solver* h, pdlpx_result* out) {
    if (h == nullptr || out == nullptr) return PDLPX_E_INVALID;
    return guarded(h, [&] { return h->engine.solve(out); });
}

int32_t pdlpx_get_status(const pdlpx_solver* h, int32_t* status) {
    if (h == nullptr || status == nullptr) return PDLPX_E_INVALID;
    *status = h->engine.status();
    return PDLPX_OK;
}

int32_t pdlpx_get_objective(const pdlpx_solver* h, double* objective) {
    if (h == nullptr || objective == nullptr) return PDLPX_E_INVALID;
    *objective = h->engine.objective();
    return PDLPX_OK;
}

int32_t pdlpx_get_primal(const pdlpx_solver* h, double* x, int32_t n) {
    if (h == nullptr || (n > 0 && x == nullptr)) return PDLPX_E_INVALID;
    const auto& v = h->engine.primal();
    if (n != static_cast<int32_t>(v.size())) return PDLPX_E_INVALID;
    if (n > 0) std::memcpy(x, v.data(), sizeof(double) * static_cast<size_t>(n));
    return PDLPX_OK;
}

int32_t pdlpx_get_dual(const pdlpx_solver* h, double* y, int32_t m) {
    if (h == nullptr || (m > 0 && y == nullptr)) return PDLPX_E_INVALID;
    const auto& v = h->engine.dual();
    if (m != static_cast<int32_t>(v.size())) return PDLPX_E_INVALID;
    if (m > 0) std::memcpy(y, v.data(), sizeof(double) * static_cast<size_t>(m));
    return PDLPX_OK;
}

int32_t pdlpx_get_reduced_costs(const pdlpx_solver* h, double* rc, int32_t n) {
    if (h == nullptr || (n > 0 && rc == nullptr)) return PDLPX_E_INVALID;
    if (n != h->engine.problem().n) return PDLPX_E_INVALID;
    return guarded(const_cast<pdlpx_solver*>(h), [&] {
        std::vector<double> v;
        h->engine.reducedCosts(v);
        if (n > 0) std::memcpy(rc, v.data(), sizeof(double) * static_cast<size_t>(n));
        return PDLPX_OK;
    });
}

int32_t pdlpx_used_gpu(const pdlpx_solver* h, int32_t* used) {
    if (h == nullptr || used == nullptr) return PDLPX_E_INVALID;
    *used = h->engine.usedGpu() ? 1 : 0;
    return PDLPX_OK;
}

int32_t pdlpx_get_dims(const pdlpx_solver* h, int32_t* m, int32_t* n, int32_t* nnz) {
    if (h == nullptr) return PDLPX_E_INVALID;
    const auto& p = h->engine.problem();
    if (m) *m = p.m;
    if (n) *n = p.n;
    if (nnz) *nnz = p.a.nnz();
    return PDLPX_OK;
}

int32_t pdlpx_add_rows(pdlpx_solver* h, int32_t rows, const int32_t* starts, const int32_t* indices,
                       const double* values, int32_t nvals, const double* lower, const double* upper) {
    if (h == nullptr) return PDLPX_E_INVALID;
    if (rows <= 0) return PDLPX_OK;
    if (starts == nullptr || lower == nullptr || upper == nullptr || (nvals > 0 && (indices == nullptr || values == nullptr)))
        return PDLPX_OK;  // the reference ignores invalid input silently
    return guarded(h, [&] {
        h->engine.addRows(rows, starts, indices, values, nvals, lower, upper);
        return PDLPX_OK;
    });
}

int32_t pdlpx_remove_rows(pdlpx_solver* h, const int32_t* rows, int32_t count) {
    if (h == nullptr) return PDLPX_E_INVALID;
    return guarded(h, [&] {
        h->engine.removeRows(rows, count);
        return PDLPX_OK;
    });
}

int32_t pdlpx_set_col_bounds(pdlpx_solver* h, int32_t col, double lower, double upper) {
    if (h == nullptr) return PDLPX_E_INVALID;
    return guarded(h, [&] {
        h->engine.setColBounds(col, lower, upper);
        return PDLPX_OK;
    });
}

int32_t pdlpx_set_objective(pdlpx_solver* h, const double* obj, int32_t n) {
    if (h == nullptr) return PDLPX_E_INVALID;
    return guarded(h, [&] {
        h->engine.setObjective(obj, n);
        return PDLPX_OK;
    });
}

int32_t pdlpx_get_scaling(const pdlpx_solver* h, double* col_scale, double* cscaled, double* col_lb_scaled,
                          double* row_scale, double* row_lb_scaled, double* row_ub_scaled, double* tau_base,
                          double* sigma_base, double* col_ub_scaled, double* objective_scale,
                          double* constraint_scale) {
    if (h == nullptr) return PDLPX_E_INVALID;
    if (!h->engine.loaded()) return PDLPX_E_NOT_LOADED;
    const auto& s = h->engine.scaled();
    auto cp = [](double* dst, const std::vector<double>& src) {
        if (dst != nullptr && !src.empty()) std::memcpy(dst, src.data(), sizeof(double) * src.size());
    };
    cp(col_scale, s.col_scale);
    cp(cscaled, s.c);
    cp(col_lb_scaled, s.cl);
    cp(col_ub_scaled, s.cu);
    cp(row_scale, s.row_scale);
    cp(row_lb_scaled, s.rl);
    cp(row_ub_scaled, s.ru);
    cp(tau_base, s.tau);
    cp(sigma_base, s.sigma);
    if (objective_scale) *objective_scale = s.obj_scale;
    if (constraint_scale) *constraint_scale = s.con_scale;
    return PDLPX_OK;
}

int32_t pdlpx_time_kernels(pdlpx_solver* h, int32_t precision, int32_t reps, int64_t flush_bytes, double* ms_primal,
                           double* ms_dual, double* ms_check) {
    if (h == nullptr) return PDLPX_E_INVALID;
    return guarded(h, [&] {
        return h->engine.timeKernels(precision, reps, flush_bytes, ms_primal, ms_dual, ms_check);
    });
}

int32_t pdlpx_get_step_times(const pdlpx_solver* h, int32_t precision, double* ms_primal, double* ms_dual,
                             int32_t* samples) {
    if (h == nullptr || (precision != PDLPX_PREC_MIXED && precision != PDLPX_PREC_FP64)) return PDLPX_E_INVALID;
    h->engine.stepTimes(precision, ms_primal, ms_dual, samples);
    return PDLPX_OK;
}

int32_t pdlpx_get_launch_config(const pdlpx_solver* h, int32_t* group_a, int32_t* group_at, int32_t* blocks_primal,
                                int32_t* blocks_dual) {
    if (h == nullptr) return PDLPX_E_INVALID;
    return h->engine.launchConfig(group_a, group_at, blocks_primal, blocks_dual);
}

int32_t pdlpx_get_long_tiles(const pdlpx_solver* h, int32_t* chunks, int32_t* groups) {
    if (h == nullptr) return PDLPX_E_INVALID;
    return h->engine.longTiles(chunks, groups);
}

int32_t pdlpx_get_hot_prefix(const pdlpx_solver* h, int32_t precision, int32_t* primal, int32_t* dual) {
    if (h == nullptr) return PDLPX_E_INVALID;
    return h->engine.hotPrefix(precision, primal, dual);
}

int32_t pdlpx_batch_solve(int32_t count, const pdlpx_lp* lps, const pdlpx_options* opts, pdlpx_result* results,
                          double* const* x_out, double* const* y_out) {
    if (count < 0 || (count > 0 && (lps == nullptr || results == nullptr))) return PDLPX_E_INVALID;
    if (count == 0) return PDLPX_OK;
    pdlpx_options o;
    if (opts)
        o = *opts;
    else
        pdlpx_options_default(&o);
    try {
        return pdlpx::batchSolve(count, lps, o, results, x_out, y_out, g_last_error);
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return PDLPX_E_NOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return PDLPX_E_INVALID;
    }
}

int32_t pdlpx_shard_lps(int32_t count, const int64_t* weights, int32_t ndev, int32_t* device_of) {
    if (count < 0 || ndev <= 0 || (count > 0 && (weights == nullptr || device_of == nullptr))) return PDLPX_E_INVALID;
    for (int32_t k = 0; k < count; ++k)
        if (weights[k] < 0) return PDLPX_E_INVALID;
    try {
        pdlpx::shardLps(count, weights, ndev, device_of);
    } catch (const std::bad_alloc&) {
        return PDLPX_E_NOMEM;
    }
    return PDLPX_OK;
}

int32_t pdlpx_batch_solve_devices(int32_t count, const pdlpx_lp* lps, const pdlpx_options* opts,
                                  const int32_t* devices, int32_t ndev, pdlpx_result* results,
                                  double* const* x_out, double* const* y_out) {
    if (count < 0 || (count > 0 && (lps == nullptr || results == nullptr)) || ndev <= 0 || devices == nullptr)
        return PDLPX_E_INVALID;
    int devcount = 0;
    if (cudaGetDeviceCount(&devcount) != cudaSuccess || devcount <= 0) {
        cudaGetLastError();
        g_last_error = "no CUDA device visible";
        return PDLPX_E_NO_DEVICE;
    }
    for (int32_t d = 0; d < ndev; ++d)
        if (devices[d] < 0 || devices[d] >= devcount) {
            g_last_error = "device ordinal " + std::to_string(devices[d]) + " out of range";
            return PDLPX_E_INVALID;
        }
    if (count == 0) return PDLPX_OK;
    pdlpx_options o;
    if (opts)
        o = *opts;
    else
        pdlpx_options_default(&o);
    try {
        return pdlpx::batchSolveDevices(count, lps, o, devices, ndev, results, x_out, y_out, g_last_error);
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return PDLPX_E_NOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return PDLPX_E_INVALID;
    }
}

int32_t pdlpx_grid_barrier_check(int32_t device, int32_t blocks, int32_t rounds, int32_t stall,
                                 int32_t* barrier_error, double* seconds) {
    if (barrier_error == nullptr || blocks < 1 || rounds < 1) return PDLPX_E_INVALID;
    try {
        return pdlpx::gridBarrierCheck(device, blocks, rounds, stall, barrier_error, seconds, g_last_error);
    } catch (const std::bad_alloc&) {
        return PDLPX_E_NOMEM;
    } catch (...) {
        return PDLPX_E_INVALID;
    }
}

int32_t pdlpx_csr_spmv(int32_t rows, int32_t cols, int32_t nnz, const int32_t* row_ptr, const int32_t* col_idx,
                       const double* val, const double* x, double* y, int32_t precision, int32_t group) {
    try {
        return pdlpx::deviceSpmv(rows, cols, nnz, row_ptr, col_idx, val, x, y, precision, group, g_last_error);
    } catch (...) {
        return PDLPX_E_INVALID;
    }
}

}  // extern "C"
