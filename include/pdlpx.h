/*
 * pdlpx.h -- C ABI of the B200-native PDLP engine (drop-in for mipx's PDLP path).
 *
 * Every entry point is plain C: opaque handles, plain pointers and sizes, int32
 * error codes (PDLPX_OK == 0), no exceptions and no torch types.  Caller buffers
 * are copied on entry (the same ownership rule as mipx::PdlpSolver::load, which
 * copies the LpProblem, src/lp/pdlp.cpp:445-455); outputs are written into
 * caller-provided host buffers.
 *
 * Reference interface each group replaces (paths inside spoorendonk/mipx):
 *   pdlpx_options            <- mipx::PdlpOptions            include/mipx/pdlp.h:19-87
 *   pdlpx_result             <- mipx::LpResult               include/mipx/lp_solver.h:11-16
 *   status codes             <- mipx::Status                 include/mipx/core.h:11-19
 *   pdlpx_create/destroy     <- PdlpSolver ctor/dtor          include/mipx/pdlp.h:89-92
 *   pdlpx_set_options        <- PdlpSolver::setOptions        include/mipx/pdlp.h:122
 *   pdlpx_load_csr           <- PdlpSolver::load(LpProblem)   include/mipx/pdlp.h:94, src/lp/pdlp.cpp:445-455
 *   pdlpx_solve              <- PdlpSolver::solve             include/mipx/pdlp.h:95, src/lp/pdlp.cpp:801-1720
 *   pdlpx_get_primal/dual    <- getPrimalValues/getDualValues include/mipx/pdlp.h:100-101, src/lp/pdlp.cpp:2800-2806
 *   pdlpx_get_reduced_costs  <- getReducedCosts               src/lp/pdlp.cpp:2808-2819
 *   pdlpx_set_warm_start     <- setWarmStart/clearWarmStart   include/mipx/pdlp.h:114-120
 *   pdlpx_set_stop_flag      <- PdlpOptions::stop_flag        include/mipx/pdlp.h:86
 *   pdlpx_set_stop_callback  <- PdlpOptions::stop_flag        include/mipx/pdlp.h:86 (any flag type)
 *   pdlpx_add_rows ...       <- addRows/removeRows/setColBounds/setObjective  src/lp/pdlp.cpp:2833-2907
 *   pdlpx_used_gpu           <- PdlpSolver::usedGpu           include/mipx/pdlp.h:124
 */
#ifndef PDLPX_H
#define PDLPX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status of a solve: same values and order as mipx::Status (core.h:11-19) ---- */
enum {
    PDLPX_STATUS_OPTIMAL = 0,
    PDLPX_STATUS_INFEASIBLE = 1,
    PDLPX_STATUS_UNBOUNDED = 2,
    PDLPX_STATUS_ITER_LIMIT = 3,
    PDLPX_STATUS_TIME_LIMIT = 4,
    PDLPX_STATUS_NODE_LIMIT = 5,
    PDLPX_STATUS_ERROR = 6
};

/* ---- error codes returned by every call ---- */
enum {
    PDLPX_OK = 0,
    PDLPX_E_INVALID = 1,     /* bad argument (null pointer, size mismatch, bad CSR) */
    PDLPX_E_NOT_LOADED = 2,  /* solve/get before load */
    PDLPX_E_CUDA = 3,        /* a CUDA runtime call failed; see pdlpx_last_error */
    PDLPX_E_NOMEM = 4,       /* device allocation failed */
    PDLPX_E_NO_DEVICE = 5,   /* no CUDA device visible */
    PDLPX_E_TIMEOUT = 6,     /* a bounded device wait ran out */
    PDLPX_E_BUSY = 7,        /* server queue full / over HBM budget */
    PDLPX_E_UNKNOWN_TICKET = 8
};

enum { PDLPX_NORM_L2 = 0, PDLPX_NORM_LINF = 1 };
enum { PDLPX_MINIMIZE = 0, PDLPX_MAXIMIZE = 1 };

/* Precision modes of the engine (no counterpart in the reference, which is FP64 only). */
enum {
    PDLPX_PREC_MIXED = 0, /* FP32 matrix/iterates/SpMV, FP64 checks, PI, objective, FP64 polish;
                             an LP whose FP64 working set per iteration is under 16 MB (L2-resident:
                             FP32 storage saves no time there) runs FP64 kernels unless fp64_switch = 0 */
    PDLPX_PREC_FP64 = 1   /* FP64 throughout ("plain FP64 GPU" mode) */
};

/* Field-for-field image of mipx::PdlpOptions (include/mipx/pdlp.h:19-87) plus engine knobs.
 * Booleans are int32 (0/1).  Call pdlpx_options_default() to get the reference defaults. */
typedef struct pdlpx_options {
    int32_t max_iter;                 /* 4000000 */
    double optimality_tol;            /* 5e-5 (relative gap) */
    double primal_tol;                /* 5e-5 */
    double dual_tol;                  /* 5e-5 */
    double max_solve_seconds;         /* -1 = no limit */
    int32_t optimality_norm;          /* PDLPX_NORM_L2 */
    int32_t sv_max_iter;              /* 5000 power iterations */
    double sv_tol;                    /* 1e-4 */
    int32_t adaptive_step;            /* 0 */
    double adaptive_step_down;        /* 0.7 */
    double adaptive_step_up;          /* 1.0 */
    double adaptive_step_min;         /* 1e-6 */
    double adaptive_step_max;         /* 1e3 */
    double primal_weight;             /* 1.0 */
    int32_t update_primal_weight;     /* 1 */
    double pid_kp;                    /* 0.99 */
    double pid_ki;                    /* 0.01 */
    double pid_kd;                    /* 0.0 */
    double pid_i_smooth;              /* 0.3 */
    double restart_sufficient_decay;  /* 0.2 */
    double restart_necessary_decay;   /* 0.5 */
    double restart_artificial_fraction; /* 0.36 */
    int32_t termination_eval_frequency; /* 200 */
    double matrix_zero_tol;           /* 0 = off */
    int32_t enable_polishing;         /* 1 */
    double polish_primal_tol;         /* 1e-6 */
    double polish_dual_tol;           /* 1e-6 */
    int32_t polish_max_iter;          /* 500000 */
    int32_t do_ruiz_scaling;          /* 1 */
    int32_t ruiz_iterations;          /* 10 */
    int32_t do_pock_chambolle_scaling;/* 1 */
    int32_t do_bound_obj_rescaling;   /* 1 */
    int32_t preconditioner_refresh;   /* 0 */
    double preconditioner_refresh_ratio; /* 10 */
    int32_t anderson_acceleration;    /* 0 */
    int32_t anderson_window_size;     /* 5 */
    double anderson_regularization;   /* 1e-10 */
    int32_t use_gpu;                  /* 1 */
    int32_t gpu_min_rows;             /* 512 (the engine always runs on the GPU; kept for parity of the struct) */
    int32_t gpu_min_nnz;              /* 10000 */
    int32_t verbose;                  /* 1 in the reference; the engine prints the same progress lines */
    /* ---- engine knobs (no counterpart in the reference) ---- */
    int32_t precision;                /* PDLPX_PREC_MIXED */
    int32_t device;                   /* CUDA device ordinal, default 0 */
    int32_t fp64_switch;              /* mixed mode: FP32 phase hands over to FP64 when its KKT stalls (1) */
    int32_t spmv_group_a;             /* 0 = autotune; else threads per row of A (1,2,4,8,16,32) */
    int32_t spmv_group_at;            /* 0 = autotune; else threads per row of A^T */
    int32_t autotune;                 /* 1: time the step kernels' launch shapes on LPs with >= 100k
                                         nonzeros and keep the fastest; in pdlpx_batch_solve and the
                                         server, time each sliced-ELL class's entries-per-round variants
                                         on the pack (identical results); 0 (default): row-length table,
                                         deterministic */
    int32_t shape_primal;             /* 0 = automatic; k > 0 pins launch shape k-1 of the primal step's
                                         short rows: 1..16 the CSR shapes (lanes x rows x loads), 17..19
                                         sliced ELL with 4 / 8 / 16 entries per round, 20..22 the same
                                         with streaming loads of the matrix (no L1 allocation,
                                         evict-first in L2; single-LP engine only) */
    int32_t shape_dual;               /* 0 = automatic; k > 0 pins launch shape k-1 of the dual step */
    int32_t batch_pack_mb;            /* pdlpx_batch_solve: device megabytes per pack of LPs solved
                                         together (0 = 85% of free device memory); larger batches are
                                         split into packs solved one after another */
    int32_t batch_compact;            /* pdlpx_batch_solve: 1 (default) drops finished LPs from the
                                         launches once they idle enough tiles; 0 never */
    int32_t batch_sell;               /* pdlpx_batch_solve: 1 (default) stores matrix sides with mean row
                                         length <= 32 as sliced ELL (32-row slices, column-major, rows
                                         sorted by length inside each 256-row tile); 0 keeps CSR */
    int32_t scale_on_device;          /* Ruiz passes of the scaling pipeline on the GPU (load, edits,
                                         batch / server preparation; identical results): -1 (default)
                                         for LPs with >= 200k nonzeros, 1 always, 0 never */
    int32_t sell;                     /* single-LP engine: store the short rows of a matrix side (rows
                                         longer than max(64, 8 x mean) excepted) as sliced ELL, 32-row
                                         slices, when their mean length is <= 64: -1 (default)
                                         automatic, 1 whenever the side has short rows, 0 never (CSR) */
    int32_t reference_fixed_columns;  /* 1: a fixed column (lb == ub) contributes to the dual residual
                                         exactly as in the reference's check (pdlp.cpp:1134-1140, lower
                                         bound tested first, so a negative reduced cost counts and
                                         such LPs may not converge, as there); 0 (default): a fixed
                                         column adds no dual residual */
    int32_t hot_cache;                /* single-LP engine, sliced-ELL sides: k > 0 serves the step's
                                         gathers of the other side's longest rows (first in the device
                                         numbering) from a shared-memory copy of that prefix held by
                                         every block, with k KB of shared memory per SM (capped at the
                                         device's limit); 0 (default) never.  Identical results either
                                         way; measured slower on the 500k x 2M power-law LP, whose
                                         popular columns L1 already caches */
    int32_t long_tiles;               /* single-LP engine, mixed mode: run the primal step of the long
                                         columns (> max(64, 8 x mean) entries) in row chunks whose FP32
                                         y sits in shared memory: -1 (default) when those columns hold
                                         at least 1.5 x SMs x chunk rows entries (a chunk: up to
                                         28,672 rows), 1 whenever there are long columns, 0 never */
    int32_t batch_persistent;         /* pdlpx_batch_solve: run the N PDHG iterations of each restart
                                         cycle as one cooperative launch over every sliced-ELL tile (a
                                         grid barrier between the primal and the dual step) instead of
                                         a graph of per-class launches: 1 on, 0 (default) off.  Packs
                                         with CSR tiles or 16-entry rounds, and the request server's
                                         packs, keep the graph.  Identical results either way */
    int32_t sell_window;              /* single-LP engine, sliced-ELL sides: the short rows are renumbered
                                         longest first inside windows of this many rows; 0 (default): one
                                         window, the whole side.  A window keeps each row within that many
                                         places of its original position (for LPs whose numbering gives
                                         the gathers locality) */
    int32_t reserved[1];
} pdlpx_options;

/* Image of mipx::LpResult (lp_solver.h:11-16) plus engine diagnostics. */
typedef struct pdlpx_result {
    int32_t status;           /* PDLPX_STATUS_* */
    double objective;         /* original space; 0 unless optimal (pdlp.cpp:1705-1709) */
    int32_t iterations;       /* PDHG iterations including polish */
    double work_units;        /* iterations * (4 nnz + 2 (m+n)), deterministic (pdlp.cpp:1716-1719) */
    /* ---- diagnostics ---- */
    double rel_primal_resid;  /* last check, reference definition (L2 or Linf per options) */
    double rel_dual_resid;
    double rel_gap;
    double primal_objective;  /* last check, original space */
    double dual_objective;
    int32_t fp64_iterations;  /* iterations run in the FP64 phase (mixed mode) */
    int32_t restarts;
    double step_size;
    double primal_weight;
    double solve_seconds;     /* wall time of pdlpx_solve */
    double device_seconds;    /* device time of the iteration loop (CUDA events) */
    int32_t used_gpu;
    int32_t kernel_launches;  /* engine kernel launches issued by this solve */
} pdlpx_result;

typedef struct pdlpx_solver pdlpx_solver; /* opaque */

/* ---- options / errors ---- */
void pdlpx_options_default(pdlpx_options* opts);
const char* pdlpx_error_string(int32_t code);
/* Last error message recorded on this handle (never NULL). */
const char* pdlpx_last_error(const pdlpx_solver* h);
/* Number of visible CUDA devices (0 on a host without a GPU; never fails). */
int32_t pdlpx_device_count(void);
/* Library version string. */
const char* pdlpx_version(void);
/* Writes sizes[0..6) = sizeof of the ABI structures as compiled into the
 * library, in the order pdlpx_options, pdlpx_result, pdlpx_lp, pdlpx_gen_lp,
 * pdlpx_server_config, pdlpx_server_stats; bindings compare their own layouts
 * against these. */
void pdlpx_struct_sizes(int32_t* sizes);

/* ---- single-LP solver (PdlpSolver : LpSolver) ---- */
int32_t pdlpx_create(const pdlpx_options* opts, pdlpx_solver** out);
int32_t pdlpx_destroy(pdlpx_solver* h);
int32_t pdlpx_set_options(pdlpx_solver* h, const pdlpx_options* opts);
int32_t pdlpx_get_options(const pdlpx_solver* h, pdlpx_options* out);
/* Load an LP in ranged form row_lb <= A x <= row_ub, col_lb <= x <= col_ub.
 * A is CSR (m rows, n cols); column indices need not be sorted; +-INFINITY (or
 * |v| >= 1e30 is NOT special-cased: pass IEEE infinities) marks absent bounds.
 * sense: PDLPX_MINIMIZE / PDLPX_MAXIMIZE.  Clears any warm start (pdlp.h:117). */
int32_t pdlpx_load_csr(pdlpx_solver* h, int32_t m, int32_t n, int32_t nnz,
                       const int32_t* row_ptr, const int32_t* col_idx, const double* val,
                       const double* obj, const double* col_lb, const double* col_ub,
                       const double* row_lb, const double* row_ub,
                       int32_t sense, double obj_offset);
/* Warm start in original space; silently ignored at solve time when the sizes
 * do not match the loaded problem (pdlp.cpp:918-919). */
int32_t pdlpx_set_warm_start(pdlpx_solver* h, const double* x, int32_t nx,
                             const double* y, int32_t ny);
int32_t pdlpx_clear_warm_start(pdlpx_solver* h);
/* Cooperative cancel: *flag != 0 makes the solve return ITER_LIMIT at the next
 * batch boundary (pdlp.cpp:972-976).  NULL clears.  Read with an atomic load. */
int32_t pdlpx_set_stop_flag(pdlpx_solver* h, const int32_t* flag);
/* Cooperative cancel through a caller function: poll(ctx) != 0 makes the solve
 * return ITER_LIMIT at the next batch boundary, like the flag above.  This is
 * how a caller maps a flag of its own type -- the reference's
 * `const std::atomic<bool>* stop_flag` (pdlp.h:86) -- without a mirroring
 * thread: poll loads the atomic.  poll runs on the thread that called
 * pdlpx_solve, once per restart cycle; it must not call back into the same
 * handle.  poll == NULL clears.  Flag and callback may both be set; either stops. */
typedef int32_t (*pdlpx_stop_poll)(void* ctx);
int32_t pdlpx_set_stop_callback(pdlpx_solver* h, pdlpx_stop_poll poll, void* ctx);
int32_t pdlpx_solve(pdlpx_solver* h, pdlpx_result* out);
int32_t pdlpx_get_status(const pdlpx_solver* h, int32_t* status);
int32_t pdlpx_get_objective(const pdlpx_solver* h, double* objective);
/* Copy the last solution (original space) into x[0..n) / y[0..m). */
int32_t pdlpx_get_primal(const pdlpx_solver* h, double* x, int32_t n);
int32_t pdlpx_get_dual(const pdlpx_solver* h, double* y, int32_t m);
int32_t pdlpx_get_reduced_costs(const pdlpx_solver* h, double* rc, int32_t n);
int32_t pdlpx_used_gpu(const pdlpx_solver* h, int32_t* used);
int32_t pdlpx_get_dims(const pdlpx_solver* h, int32_t* m, int32_t* n, int32_t* nnz);
/* Incremental edits; each re-runs the scaling pipeline like the reference.
 * Invalid input is ignored silently (pdlp.cpp:2841-2853). */
int32_t pdlpx_add_rows(pdlpx_solver* h, int32_t rows, const int32_t* starts,
                       const int32_t* indices, const double* values, int32_t nvals,
                       const double* lower, const double* upper);
int32_t pdlpx_remove_rows(pdlpx_solver* h, const int32_t* rows, int32_t count);
int32_t pdlpx_set_col_bounds(pdlpx_solver* h, int32_t col, double lower, double upper);
int32_t pdlpx_set_objective(pdlpx_solver* h, const double* obj, int32_t n);

/* Scaled problem as the engine prepared it (for parity of the scaling pipeline
 * with pdlp.cpp:469-669).  Any output pointer may be NULL.  Sizes: n, n, n, m, m, m, n, m, n. */
int32_t pdlpx_get_scaling(const pdlpx_solver* h, double* col_scale, double* cscaled,
                          double* col_lb_scaled, double* row_scale, double* row_lb_scaled,
                          double* row_ub_scaled, double* tau_base, double* sigma_base,
                          double* col_ub_scaled, double* objective_scale,
                          double* constraint_scale);

/* Average device time in milliseconds of one launch of the fused primal step
 * and the fused dual step (each with its long- and short-row launches) in the
 * given precision (PDLPX_PREC_MIXED: the FP32 kernels, PDLPX_PREC_FP64: the
 * FP64 kernels; -1: the precision the last solve ended in), run as `reps`
 * PDHG iterations -- primal, dual, primal, ... as in the solve loop -- with a
 * CUDA event between every two launches on the engine's stream, after a write
 * of flush_bytes bytes to a scratch buffer (0: none) that evicts the L2; and
 * of one FP64 check pass.  Needs a completed pdlpx_solve on this handle and, for
 * PDLPX_PREC_MIXED, a mixed-precision image; leaves the returned solution
 * untouched.  Any output pointer may be NULL. */
int32_t pdlpx_time_kernels(pdlpx_solver* h, int32_t precision, int32_t reps, int64_t flush_bytes,
                           double* ms_primal, double* ms_dual, double* ms_check);
/* Device time of the step kernels measured inside the last solve itself: the
 * restart-cycle graph records CUDA events around the primal and the dual step
 * of one iteration of every cycle, and the host reads them after the cycle.
 * For precision p (PDLPX_PREC_MIXED: FP32 kernels, PDLPX_PREC_FP64: FP64
 * kernels) returns the mean ms per launch of each step and the number of
 * cycles sampled (0: none ran in that precision). */
int32_t pdlpx_get_step_times(const pdlpx_solver* h, int32_t precision, double* ms_primal, double* ms_dual,
                             int32_t* samples);
/* Threads per row chosen for A (dual step) and A^T (primal step) -- 1 for a
 * side stored as sliced ELL -- and the grid sizes of the two step kernels'
 * short-row launches. */
int32_t pdlpx_get_launch_config(const pdlpx_solver* h, int32_t* group_a, int32_t* group_at,
                                int32_t* blocks_primal, int32_t* blocks_dual);
/* Length of the hot prefix (option hot_cache) that the primal step's gathers
 * of y and the dual step's gathers of x serve from shared memory, at the
 * given precision (PDLPX_PREC_MIXED: the FP32 kernels; PDLPX_PREC_FP64);
 * 0 where that step runs without one. */
int32_t pdlpx_get_hot_prefix(const pdlpx_solver* h, int32_t precision, int32_t* primal, int32_t* dual);
/* Row chunks and column groups of the tiled long-column primal step (option
 * long_tiles) of the loaded LP; 0 chunks where the CSR launch runs. */
int32_t pdlpx_get_long_tiles(const pdlpx_solver* h, int32_t* chunks, int32_t* groups);

/* ---- batched solve: many independent LPs in one persistent launch ---- */
typedef struct pdlpx_lp {
    int32_t m, n, nnz;
    const int32_t* row_ptr;
    const int32_t* col_idx;
    const double* val;
    const double* obj;
    const double* col_lb;
    const double* col_ub;
    const double* row_lb;
    const double* row_ub;
    int32_t sense;
    double obj_offset;
    const double* warm_x; /* optional (NULL) */
    const double* warm_y; /* optional (NULL) */
} pdlpx_lp;

/* Solve count LPs with one option set.  results[count]; x_out[k] / y_out[k] may be
 * NULL or point to n_k / m_k doubles. */
int32_t pdlpx_batch_solve(int32_t count, const pdlpx_lp* lps, const pdlpx_options* opts,
                          pdlpx_result* results, double* const* x_out, double* const* y_out);

/* ---- several GPUs: independent LPs sharded across devices ----
 * No counterpart in the reference.  pdlpx_shard_lps assigns count LPs of the
 * given non-negative weights to ndev devices by longest-processing-time bin
 * packing: heaviest first, each onto the device with the least weight so far
 * (ties to the lower device index, equal weights in input order), so the
 * assignment is deterministic and balanced to within one LP's weight.
 * device_of[count] receives indices in [0, ndev). */
int32_t pdlpx_shard_lps(int32_t count, const int64_t* weights, int32_t ndev, int32_t* device_of);
/* pdlpx_batch_solve over the CUDA devices devices[0..ndev): the LPs are
 * sharded by per-iteration work (nnz + m + n) with pdlpx_shard_lps and each
 * device solves its share with its own host thread, stream and packs; no data
 * moves between devices and no collective runs.  Repeated ordinals are allowed
 * (the shares then run side by side on one device).  Results as
 * pdlpx_batch_solve, each identical to that LP's single-device result. */
int32_t pdlpx_batch_solve_devices(int32_t count, const pdlpx_lp* lps, const pdlpx_options* opts,
                                  const int32_t* devices, int32_t ndev, pdlpx_result* results,
                                  double* const* x_out, double* const* y_out);

/* The grid barrier of the persistent batch cycle (option batch_persistent) run
 * on its own: `rounds` barriers over `blocks` cooperative blocks of one warp on
 * `device`.  No counterpart in the reference.  Each block waits on the
 * barrier's generation word for at most 2^22 polls of a 64 ns sleep (about
 * 0.3-1 s); a block that runs out sets the error word and returns, and so does
 * every other block at its next barrier.  stall != 0 preloads the arrival
 * count so that no barrier completes: every block runs out.  Returns PDLPX_OK
 * when every barrier completed, PDLPX_E_TIMEOUT when one ran out (the status
 * pdlpx_batch_solve returns then), PDLPX_E_INVALID when the blocks do not fit
 * one cooperative wave; *barrier_error receives the error word and *seconds
 * (may be NULL) the launch's device time. */
int32_t pdlpx_grid_barrier_check(int32_t device, int32_t blocks, int32_t rounds, int32_t stall,
                                 int32_t* barrier_error, double* seconds);

/* ---- request server: LP solves as they arrive, continuously batched ----
 * No counterpart in the reference (the MIP search there calls PdlpSolver::solve
 * once per LP).  Submitted LPs are copied and scaled by a pool of host threads,
 * then packed with whatever else is waiting into packs solved by the batched
 * engine, several packs at a time on their own CUDA streams, within a device
 * memory budget; a request that arrives while packs run starts in the next
 * pack as soon as a stream and memory are free, and each LP's result is
 * available as soon as the restart cycle that finishes it returns.  An LP's
 * result does not depend on what it was packed with (bit-identical alone and
 * in any mix, same options); a family member's result does not depend on the
 * other members of its family pack. */
typedef struct pdlpx_server pdlpx_server;

typedef struct pdlpx_server_config {
    double budget_bytes;   /* device bytes of the packs in flight; 0 = 85% of free memory */
    int32_t max_packs;     /* packs solved at the same time (streams), default 4 */
    int32_t max_pack_lps;  /* LPs per pack, default 32 */
    int32_t prep_threads;  /* host threads scaling submitted LPs, 0 = all cores but one (pack threads
                              sleep while their restart cycles run) */
    int32_t queue_limit;   /* unfinished requests before submit returns PDLPX_E_BUSY, default 100000 */
    int32_t batch_window_ms; /* a pack starts when max_pack_lps requests are ready or the oldest ready
                                request has waited this long (default 50; 0 = start at once) */
    int32_t families;      /* 1 (default): a request submitted with a warm-start ticket whose rows begin
                              with the ticket's rows unchanged (a branch-and-bound node: new bounds,
                              appended rows) is solved in a family pack with the other nodes of that
                              ticket -- the shared rows stored once, FP64 iterates; 0: regular packs */
    int32_t num_devices;   /* 0 or 1: packs run on opts->device; k in 2..16: packs are placed on the
                              CUDA devices devices[0..k), each pack on the listed device with a free
                              stream and the fewest bytes in flight (max_packs streams and its own
                              budget per device; no data moves between devices) */
    int32_t lane_admission; /* 1 (default): a family member that arrives while a family pack of its
                               family runs takes a free lane of that pack between restart cycles
                               (the lane of a finished member, or an unused one); 0: it waits for
                               a new pack */
    int32_t devices[16];
} pdlpx_server_config;

typedef struct pdlpx_server_stats {
    int64_t submitted, completed; /* requests */
    int64_t waiting;              /* submitted, not yet in a running pack */
    int64_t running;              /* in a running pack */
    int32_t packs_running, reserved0;
    double p50_latency_s, p99_latency_s, mean_latency_s, max_latency_s; /* submit -> result */
    double lps_per_sec;           /* completed / (last completion - first submission) */
    double bytes_in_flight;       /* device bytes of the running packs */
    int64_t admitted;             /* requests that joined a running family pack in a free lane */
} pdlpx_server_stats;

void pdlpx_server_config_default(pdlpx_server_config* c);
int32_t pdlpx_server_create(const pdlpx_options* opts, const pdlpx_server_config* cfg, pdlpx_server** out);
/* Stops the running packs between restart cycles (their unfinished requests end
 * with status TimeLimit), joins the threads and frees everything. */
int32_t pdlpx_server_destroy(pdlpx_server* s);
/* Copies the LP (and its warm start, if both warm_x and warm_y are given). */
int32_t pdlpx_server_submit(pdlpx_server* s, const pdlpx_lp* lp, int64_t* ticket);
/* Warm start from a finished, unreleased request: its x when the sizes match,
 * its y for the first rows (rows beyond it, e.g. appended cuts, start at 0). */
int32_t pdlpx_server_submit_warm(pdlpx_server* s, const pdlpx_lp* lp, int64_t warm_ticket, int64_t* ticket);
int32_t pdlpx_server_poll(pdlpx_server* s, int64_t ticket, int32_t* done);
/* Waits up to timeout_seconds (< 0: no limit); PDLPX_E_TIMEOUT if unfinished. */
int32_t pdlpx_server_wait(pdlpx_server* s, int64_t ticket, double timeout_seconds, pdlpx_result* out);
int32_t pdlpx_server_get_solution(const pdlpx_server* s, int64_t ticket, double* x, int32_t n, double* y,
                                  int32_t m);
/* Forgets a finished request (its solution can no longer be read or warm-start another). */
int32_t pdlpx_server_release(pdlpx_server* s, int64_t ticket);
int32_t pdlpx_server_get_stats(const pdlpx_server* s, pdlpx_server_stats* out);
const char* pdlpx_server_last_error(const pdlpx_server* s);

/* ---- device kernels exposed for parity tests (host buffers in and out) ---- */
/* y = A x with the engine's SpMV kernel.  precision: PDLPX_PREC_MIXED (FP32 values,
 * FP32 x, FP32 accumulation) or PDLPX_PREC_FP64.  group: threads per row (0 = auto). */
int32_t pdlpx_csr_spmv(int32_t rows, int32_t cols, int32_t nnz, const int32_t* row_ptr,
                       const int32_t* col_idx, const double* val, const double* x, double* y,
                       int32_t precision, int32_t group);

/* Row violation of a point x against ranged rows, FP64 on the device (host
 * buffers in and out): v_i = (A x)_i - clamp((A x)_i, row_lb_i, row_ub_i),
 * *sum_sq = sum_i v_i^2, *max_abs = max_i |v_i|.  This is the primal-residual
 * reduction of the convergence check (pdlp.cpp:1106-1117) exposed on its own;
 * the reduction order is fixed, so repeated calls return identical values. */
int32_t pdlpx_row_violation(int32_t m, int32_t n, int32_t nnz, const int32_t* row_ptr,
                            const int32_t* col_idx, const double* val, const double* x,
                            const double* row_lb, const double* row_ub, double* sum_sq,
                            double* max_abs);

/* Same reduction for callers that cannot allocate device memory (code running
 * inside another framework's memory pool or under an allocation-free policy).
 * No counterpart in the reference.  All pointers are DEVICE pointers; the result
 * (sum_sq, max_abs) is written to d_out[0..1] on `stream` (a cudaStream_t, NULL =
 * the legacy default stream); synchronise before reading it.  The call allocates
 * nothing: the per-block partials live in a fixed 64 KiB device array that every
 * GPU loading the library holds until exit.  Limit: at most 4096 blocks of 256
 * threads, i.e. m * G <= 1048576 where G is the threads per row chosen from the
 * mean row length nnz/m (1 up to 3, 2 up to 6, 4 up to 12, 8 up to 24, 16 up to
 * 48, 32 up to 128, 64 up to 384, 128 up to 768, else 256); larger inputs return
 * PDLPX_E_INVALID with the reason in pdlpx_last_error(NULL).  The first call on
 * each device resolves the array's device address with that device current;
 * make that first call before any stream capture.  The cached address belongs
 * to the device's current context: after cudaDeviceReset on that device it is
 * stale and the library must not be called on that device again in the same
 * process.  Calls share the array and race if they overlap on the GPU. */
int32_t pdlpx_row_violation_noalloc(int32_t m, int32_t n, int32_t nnz, const int32_t* d_row_ptr,
                                    const int32_t* d_col_idx, const double* d_val,
                                    const double* d_x, const double* d_row_lb,
                                    const double* d_row_ub, double* d_out, void* stream);

/* ---- seeded synthetic LP generators (configs of the benchmark suite) ----
 * Output arrays are allocated by the library and released with pdlpx_free_lp. */
typedef struct pdlpx_gen_lp {
    int32_t m, n, nnz;
    int32_t* row_ptr;
    int32_t* col_idx;
    double* val;
    double* obj;
    double* col_lb;
    double* col_ub;
    double* row_lb;
    double* row_ub;
    double* x0;        /* feasible point used by the construction (length n), NULL from pdlpx_read_mps */
    int32_t* is_int;   /* integrality marks (length n) or NULL */
    double obj_offset; /* objective constant (0 for the generators) */
} pdlpx_gen_lp;

/* Random sparse LP: columns with U{nnz_lo..nnz_hi} nonzeros at uniform rows,
 * values N(0,1) (duplicates summed), x0~U[0,10], rows alternate '=' and '<='
 * with b = A x0 (+U[0,1] slack on '<='), 0<=x<=10, c~N(0,1). */
int32_t pdlpx_gen_random(int32_t m, int32_t n, int32_t nnz_lo, int32_t nnz_hi, uint64_t seed,
                         pdlpx_gen_lp* out);
/* Transportation LP: s supplies x d demands, costs U[1,100], supplies U[50,150],
 * demands U[50,150] rescaled to total 0.95 * total supply. */
int32_t pdlpx_gen_transport(int32_t s, int32_t d, uint64_t seed, pdlpx_gen_lp* out);
/* Large LP: power-law column counts (min 2, max kmax, mean kmean), values N(0,1),
 * a fraction big_frac of rows scaled by big_scale, random-LP feasibility construction. */
int32_t pdlpx_gen_powerlaw(int32_t m, int32_t n, int32_t kmin, int32_t kmax, double kmean,
                           double big_frac, double big_scale, uint64_t seed, pdlpx_gen_lp* out);
void pdlpx_free_lp(pdlpx_gen_lp* lp);

/* Read an LP from a free-format MPS file, plain or gzip-compressed, with the
 * meaning mipx's reader gives every section (readMps, src/io/mps_reader.cpp:432-813):
 * N/L/G/E rows, integer markers, objective constant = -(RHS of the objective
 * row), RANGES, bounds LO/UP/FX/FR/MI/PL/BV/LI/UI/SC/SI, columns defaulting to
 * [0, +inf), minimisation; rows' entries sorted, duplicates summed, zeros
 * dropped.  Output allocated by the library (release with pdlpx_free_lp);
 * is_int marks integer columns (the LP ignores them).  Errors: PDLPX_E_INVALID
 * with the file position in pdlpx_last_error(NULL). */
int32_t pdlpx_read_mps(const char* path, pdlpx_gen_lp* out);

#ifdef __cplusplus
}
#endif

#endif /* PDLPX_H */
