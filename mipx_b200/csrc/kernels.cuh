// Device code of the PDLP engine (sm_100a).
//
// One PDHG iteration is two fused kernels:
//   primalStep : (A^T y_cur)_j computed by a G-lane group on row j of A^T,
//                then the Halpern primal step of column j in the same thread
//                (pdlp_kernels.cu:46-88 restated around a fused SpMV).
//   dualStep   : (A x_refl)_i by a G-lane group on row i of A, then the dual
//                proximal step of row i (pdlp_kernels.cu:94-157).
// so the SpMV results never go to memory.  Every N iterations a check pass
// (checkRows, checkCols) evaluates in FP64 everything the controller needs --
// KKT residuals, objectives, fixed-point error, PI distances and the
// infeasibility / unboundedness certificate tests -- as deterministic
// per-block partials, and the single-block controller reduces them in fixed
// order and runs the restart / primal-weight / polish / termination logic of
// PdlpSolver::solve (pdlp.cpp:2196-2469, 2474-2676) on the device, so a whole
// restart cycle is one CUDA graph with no host round trip inside.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <math_constants.h>

namespace pdlpx {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;

// ---------------------------------------------------------------------------
// Device-resident state of one LP solve.
// ---------------------------------------------------------------------------
struct DevState {
    double step;  // step size (0.998 / ||A||_2)
    double pw;    // primal weight omega
    float tau_fac;  // float(step / pw), FP32 primal step factor
    float sig_fac;  // float(step * pw), FP32 dual step factor
    int inner;      // Halpern inner count at the start of the running batch
    int total;      // iterations done (main + polish)
    int polish_count;
    int done;       // 1: finished, every kernel returns at entry
    int status;     // PDLPX_STATUS_* once done
    int phase;      // 0: main loop, 1: feasibility polish
    int restart;    // controller verdict of the last check: copy pdhg -> initial/current
    int prec;       // iterate precision in use: 0 FP32, 1 FP64
    int promote;    // controller asks for the FP32 -> FP64 hand-over
    int converged;  // main loop met its tolerances
    int restarts;
    int checks;
    int stall;      // checks since the best KKT score improved (mixed mode)
    int have_prev;  // adaptive step: previous check stored
    int cert_hit;   // 1 infeasible certificate, 2 unbounded certificate
    int switch_total;  // iteration count at the FP32 -> FP64 hand-over (-1: none)
    double fpe0, last_fpe;   // restart bookkeeping (initial_fpe / last_trial_fpe)
    double esum, elast;      // PI controller integral / last error
    double best_pw, best_score;
    double best_kkt;
    double precond_pw;
    // last check, original space
    double rel_p, rel_d, rel_pi, rel_di, gap, pobj, dobj, fpe, pterm, dterm;
};

// Per-solve constants of the controller.
struct DevConst {
    int m, n, N;
    int max_iter, polish_max_iter;
    int linf, update_pw, enable_polish, mixed, fp64_switch, adaptive, precond_refresh;
    int nb_rows, nb_cols;  // number of check partial blocks
    int stall_limit;
    int ref_fixed;         // 1: a fixed column's dual residual as in the reference's check
    double primal_tol, dual_tol, opt_tol, polish_ptol, polish_dtol;
    double kp, ki, kd, ismooth, suff, nec, art;
    double c_norm, b_norm, obj_sign, obj_scale, con_scale, offset;
    double step_lb, step_ub, step_down, step_up;
    double precond_ratio;
    double switch_score;
    double noise_factor;  // hand-over only when a residual is within this factor of its FP32 noise floor
};

// Packed per-column / per-row constants of the step kernels (one vector load each).
template <class T>
struct ColPack;
template <>
struct __align__(16) ColPack<float> {
    float c, lb, ub, tau;
};
template <>
struct __align__(32) ColPack<double> {
    double c, lb, ub, tau;
};
template <class T>
struct RowPack;
template <>
struct __align__(16) RowPack<float> {
    float sigma, rl, ru, type;
};
template <>
struct __align__(32) RowPack<double> {
    double sigma, rl, ru, type;
};

template <class T>
struct IterArgs {
    const int* __restrict__ at_ptr;
    const int* __restrict__ at_idx;
    const T* __restrict__ at_val;
    const int* __restrict__ a_ptr;
    const int* __restrict__ a_idx;
    const T* __restrict__ a_val;
    const ColPack<T>* __restrict__ cp;
    const RowPack<T>* __restrict__ rp;
    // The current iterates carry the Halpern state from one iteration to the
    // next and stay FP64 in every mode: rounding them to FP32 on each store is
    // a random walk of ~sqrt(K) * 6e-8 over K iterations, which stalled a
    // 1M-variable transportation LP at 1e-4 relative primal residual.
    double* xc;  // current x
    T* xi;       // initial (anchor) x
    T* xr;       // reflected x (gathered by the dual SpMV)
    T* xh;       // pdhg x (written on the last iteration of a batch)
    double* yc;  // current y
    T* yi;
    T* yh;
    DevState* st;
    int m, n;
    int max_iter, polish_max_iter, N;
    // y as the single-LP engine's primal SpMV gathers it (kernels with YG):
    // an FP32 copy of yc kept by every writer of yc in mixed mode -- its
    // rounding is of the order of the FP32 matrix values' own, and a 4-byte
    // gather costs the L1 tag stage half of an 8-byte one -- and yc itself in
    // FP64 mode.  Null elsewhere (the packed batch gathers yc).
    T* yg = nullptr;
};

// Row / column metric slots of the check pass.
enum RowSlot {
    R_PRES_SQ = 0,  // sum  |A x - proj(A x)|^2 (original units)
    R_PRES_MAX,     // max
    R_DOBJ_ROW,     // sum  row support term of the dual objective
    R_DDIST,        // sum  (y_hat - y_init)^2
    R_YNORM,        // sum  (y_hat * row_scale)^2           certificate
    R_MIN_LE,       // min  over '<=' rows of s*y*r           certificate
    R_MAX_GE,       // max  over '>=' rows                     certificate
    R_FARKAS_ROW,   // sum  s*y * selected row bound (scaled)  certificate
    R_UB_TWO,       // max  |Ax/r| over two-sided rows          certificate
    R_UB_LE,        // max  Ax/r over '<=' rows                 certificate
    R_UB_GE,        // min  Ax/r over '>=' rows                 certificate
    R_ADAPT,        // sum  sigma_i (Ax - prev Ax)^2           adaptive step
    R_NOISE_SQ,     // sum  (sum_j |a_ij x_j|)^2 (original units)  FP32 noise floor of the primal residual
    kRowSlots
};
enum ColSlot {
    C_POBJ = 0,   // sum c x
    C_DRES_SQ,    // sum dual residual^2 (original units)
    C_DRES_MAX,   // max
    C_DOBJ_COL,   // sum column support term
    C_PDIST,      // sum (x_hat - x_init)^2
    C_INTER,      // sum (A^T dy)_j (x_hat - x_init)_j
    C_XNORM,      // sum (x_hat * col_scale)^2              certificate
    C_MIN_XLB,    // min over finite-lb columns of x*cs     certificate
    C_MAX_XUB,    // max over finite-ub columns             certificate
    C_MIN_GLB,    // min over finite-lb columns of s*(A^T y)/cs  certificate
    C_MAX_GUB,    // max over finite-ub columns                  certificate
    C_COLSUP,     // sum column support of the dual ray         certificate
    C_ADAPT,      // sum (x_hat - prev x_hat)^2 / tau        adaptive step
    C_NOISE_SQ,   // sum (sum_i |a_ij y_i|)^2 (original units)   FP32 noise floor of the dual residual
    kColSlots
};
enum SlotOp { OP_SUM = 0, OP_MIN = 1, OP_MAX = 2 };

__host__ __device__ constexpr int rowSlotOp(int s) {
    return (s == R_PRES_MAX || s == R_MAX_GE || s == R_UB_TWO || s == R_UB_LE) ? OP_MAX
           : (s == R_MIN_LE || s == R_UB_GE)                                  ? OP_MIN
                                                                              : OP_SUM;
}
__host__ __device__ constexpr int colSlotOp(int s) {
    return (s == C_DRES_MAX || s == C_MAX_XUB || s == C_MAX_GUB) ? OP_MAX
           : (s == C_MIN_XLB || s == C_MIN_GLB)                  ? OP_MIN
                                                                 : OP_SUM;
}

template <class T>
struct CheckArgs {
    const int* __restrict__ a_ptr;
    const int* __restrict__ a_idx;
    const double* __restrict__ a_val;
    const int* __restrict__ at_ptr;
    const int* __restrict__ at_idx;
    const double* __restrict__ at_val;
    const T* xh;
    const T* xi;
    const T* yh;
    const T* yi;
    const double* __restrict__ c64;
    const double* __restrict__ lb64;
    const double* __restrict__ ub64;
    const double* __restrict__ cs64;  // col_scale
    const double* __restrict__ tau64; // tau_base (adaptive step)
    const double* __restrict__ rl64;
    const double* __restrict__ ru64;
    const double* __restrict__ rs64;  // row_scale
    const double* __restrict__ sig64; // sigma_base (adaptive step)
    double* prev_ax;   // adaptive step history (may be null)
    double* prev_xh;
    double* part_rows;  // [nb_rows][kRowSlots]
    double* part_cols;  // [nb_cols][kColSlots]
    const DevConst* dc;
    DevState* st;
    int m, n;
};

// ---------------------------------------------------------------------------
// Group reductions.  A G-lane group (G a power of two) owns one matrix row.
// ---------------------------------------------------------------------------
template <int G, class T>
__device__ __forceinline__ T groupSum(T s) {
    if constexpr (G == 1) {
        return s;
    } else if constexpr (G <= 32) {
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off, G);
        return s;
    } else {
        __shared__ T red[kWarps];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        const int warp = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) red[warp] = s;
        __syncthreads();
        constexpr int W = G / 32;
        const int g0 = (warp / W) * W;
        T t = red[g0];
#pragma unroll
        for (int w = 1; w < W; ++w) t += red[g0 + w];
        __syncthreads();
        return t;
    }
}

// Partial dot product of one CSR row against a gathered vector.  Lane-strided;
// every round issues U index/value loads per lane together (predicated, so a
// row whose length is not a multiple of U*G has no sequential tail), then the U
// gathers.  A masked slot gathers x[0], which exists whenever the row is
// non-empty.  FP32 data accumulate in FP64: a float*float product is exact in
// double, so the only rounding left is that of the stored operands.
template <int G, int U, class Acc, class V, class X>
__device__ __forceinline__ Acc rowDotU(int b, int e, int lane, const int* __restrict__ idx,
                                       const V* __restrict__ val, const X* __restrict__ x) {
    Acc s[U];
#pragma unroll
    for (int u = 0; u < U; ++u) s[u] = Acc(0);
    for (int k0 = b + lane; k0 < e; k0 += U * G) {
        int c[U];
        V v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + u * G;
            const bool ok = k < e;
            c[u] = ok ? __ldg(idx + k) : 0;
            v[u] = ok ? __ldg(val + k) : V(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) s[u] += static_cast<Acc>(v[u]) * static_cast<Acc>(__ldg(x + c[u]));
    }
    Acc t = s[0];
#pragma unroll
    for (int u = 1; u < U; ++u) t += s[u];
    return t;
}

template <int G, class Acc, class V, class X>
__device__ __forceinline__ Acc rowDot(int b, int e, int lane, const int* __restrict__ idx,
                                      const V* __restrict__ val, const X* __restrict__ x) {
    return rowDotU<G, 4, Acc>(b, e, lane, idx, val, x);
}

// rowDot (same loads, same accumulation order for the dot product) that also
// sums |a_k x_k|: the scale of the rounding an FP32 product of this row carries.
template <int G, class V, class X>
__device__ __forceinline__ double rowDotAbs(int b, int e, int lane, const int* __restrict__ idx,
                                            const V* __restrict__ val, const X* __restrict__ x, double& sa) {
    constexpr int U = 4;
    double s[U], a[U];
#pragma unroll
    for (int u = 0; u < U; ++u) s[u] = a[u] = 0.0;
    for (int k0 = b + lane; k0 < e; k0 += U * G) {
        int c[U];
        V v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + u * G;
            const bool ok = k < e;
            c[u] = ok ? __ldg(idx + k) : 0;
            v[u] = ok ? __ldg(val + k) : V(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const double p = static_cast<double>(v[u]) * static_cast<double>(__ldg(x + c[u]));
            s[u] += p;
            a[u] += fabs(p);
        }
    }
    double t = s[0];
    sa = a[0];
#pragma unroll
    for (int u = 1; u < U; ++u) {
        t += s[u];
        sa += a[u];
    }
    return t;
}

// Two dot products of one row (A^T y and A^T (y - y0)) in one pass, and the
// sum of |a_k y_k| (the scale of the rounding an FP32 product of the row carries).
template <int G>
__device__ __forceinline__ void rowDot2(int b, int e, int lane, const int* __restrict__ idx,
                                        const double* __restrict__ val, const float* y,
                                        const float* y0, double& s, double& d, double& sa) {
    double a0 = 0, a1 = 0, b0 = 0, b1 = 0, z0 = 0, z1 = 0;
    int k = b + lane;
    for (; k + G < e; k += 2 * G) {
        const int c0 = __ldg(idx + k), c1 = __ldg(idx + k + G);
        const double v0 = __ldg(val + k), v1 = __ldg(val + k + G);
        const double y0v = y[c0], y1v = y[c1];
        a0 += v0 * y0v;
        a1 += v1 * y1v;
        z0 += fabs(v0 * y0v);
        z1 += fabs(v1 * y1v);
        b0 += v0 * (y0v - static_cast<double>(y0[c0]));
        b1 += v1 * (y1v - static_cast<double>(y0[c1]));
    }
    for (; k < e; k += G) {
        const int c = __ldg(idx + k);
        const double v = __ldg(val + k), yv = y[c];
        a0 += v * yv;
        z0 += fabs(v * yv);
        b0 += v * (yv - static_cast<double>(y0[c]));
    }
    s = a0 + a1;
    d = b0 + b1;
    sa = z0 + z1;
}
template <int G>
__device__ __forceinline__ void rowDot2(int b, int e, int lane, const int* __restrict__ idx,
                                        const double* __restrict__ val, const double* y,
                                        const double* y0, double& s, double& d, double& sa) {
    double a0 = 0, a1 = 0, b0 = 0, b1 = 0, z0 = 0, z1 = 0;
    int k = b + lane;
    for (; k + G < e; k += 2 * G) {
        const int c0 = __ldg(idx + k), c1 = __ldg(idx + k + G);
        const double v0 = __ldg(val + k), v1 = __ldg(val + k + G);
        const double y0v = y[c0], y1v = y[c1];
        a0 += v0 * y0v;
        a1 += v1 * y1v;
        z0 += fabs(v0 * y0v);
        z1 += fabs(v1 * y1v);
        b0 += v0 * (y0v - y0[c0]);
        b1 += v1 * (y1v - y0[c1]);
    }
    for (; k < e; k += G) {
        const int c = __ldg(idx + k);
        const double v = __ldg(val + k), yv = y[c];
        a0 += v * yv;
        z0 += fabs(v * yv);
        b0 += v * (yv - y0[c]);
    }
    s = a0 + a1;
    d = b0 + b1;
    sa = z0 + z1;
}

__device__ __forceinline__ bool active(const DevState* st, int prec, int koff, int max_iter,
                                       int polish_max_iter, bool& last, int N) {
    if (st->done || st->prec != prec) return false;
    const int cur = st->phase == 0 ? st->total : st->polish_count;
    const int lim = st->phase == 0 ? max_iter : polish_max_iter;
    if (cur + koff > lim) return false;
    last = (koff == N) || (cur + koff == lim);
    return true;
}

template <class T>
__host__ __device__ constexpr int precTag() {
    return sizeof(T) == 8 ? 1 : 0;
}

// Launch shapes of the step kernels: G lanes per row, R rows per group (rows
// r*slab apart so every load instruction is coalesced across the block), U
// loads per lane per round.  The table is the autotuner's search space.
struct StepShape {
    int G, R, U;
};
constexpr StepShape kShapes[] = {
    {1, 1, 2}, {1, 2, 2}, {1, 4, 2}, {2, 1, 2}, {2, 2, 2}, {4, 1, 4}, {4, 2, 4}, {8, 1, 4},
    {16, 1, 4}, {32, 1, 4}, {32, 1, 8}, {64, 1, 4}, {64, 1, 8}, {128, 1, 8}, {256, 1, 4}, {256, 1, 8},
};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

// Halpern primal step of column j given s = (A^T y_cur)_j: projected gradient
// step, reflection, averaging with the anchor (pdlp_kernels.cu:46-88).  FP64
// arithmetic with the reference's association (tau = step * tau_base / omega).
template <class T>
__device__ __forceinline__ void primalUpdate(const IterArgs<T>& p, int j, const ColPack<T>& q, double xcd, double xid,
                                             double s, double step, double pw, double lam, bool last) {
    const double tau = step * static_cast<double>(q.tau) / pw;
    double xh = xcd - tau * (static_cast<double>(q.c) + s);
    const double lb = q.lb, ub = q.ub;
    if (xh < lb) xh = lb;
    if (xh > ub) xh = ub;
    const double xr = 2.0 * xh - xcd;
    p.xr[j] = static_cast<T>(xr);
    p.xc[j] = lam * xr + (1.0 - lam) * xid;
    if (last) p.xh[j] = static_cast<T>(xh);
}

// Dual proximal step of row i given s = (A x_refl)_i (pdlp_kernels.cu:94-157):
// the projection of y + sigma (A x_refl) by row type, reflection, averaging.
template <class T>
__device__ __forceinline__ void dualUpdate(const IterArgs<T>& p, int i, const RowPack<T>& q, double ycd, double yid,
                                           double s, double step, double pw, double lam, bool last) {
    const double sig = step * static_cast<double>(q.sigma) * pw;
    const double v = ycd + sig * s;
    const double rl = q.rl, ru = q.ru;
    const int type = static_cast<int>(q.type);
    double py;
    if (type == 0) {
        py = v - sig * rl;
    } else if (type == 1) {
        py = v - sig * ru;
        if (py < 0.0) py = 0.0;
    } else if (type == 2) {
        py = v - sig * rl;
        if (py > 0.0) py = 0.0;
    } else {
        if (v >= sig * ru)
            py = v - sig * ru;
        else if (v <= sig * rl)
            py = v - sig * rl;
        else
            py = 0.0;
    }
    const double yr = 2.0 * py - ycd;
    const double yn = lam * yr + (1.0 - lam) * yid;
    p.yc[i] = yn;
    if constexpr (sizeof(T) == 4) {
        if (p.yg != nullptr) p.yg[i] = static_cast<float>(yn);
    }
    if (last) p.yh[i] = static_cast<T>(py);
}

// Row pointers of the R rows j0 + r * slab below jend handled by one G-lane
// group (b = e = 0 past the end).
template <int G, int R>
__device__ __forceinline__ void rowBounds(const int* __restrict__ ptr, int j0, int jend, int (&b)[R], int (&e)[R]) {
    constexpr int slab = kBlock / G;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int j = j0 + r * slab;
        b[r] = 0;
        e[r] = 0;
        if (j < jend) {
            b[r] = ptr[j];
            e[r] = ptr[j + 1];
        }
    }
}

// Fused A^T y_cur + Halpern primal step (pdlp_kernels.cu:46-88 around a fused
// SpMV) of the columns j0 + r * slab (r < R) below jend, with their A^T row
// bounds already loaded.  All loads of the R columns -- packed constants,
// current / anchor x, then the A^T row entries and the y gathers -- are issued
// before the solver state is consulted, so their latencies overlap.  The step
// arithmetic is FP64 whatever the storage type (same association as the
// reference: tau = step * tau_base / omega), results are rounded once on store.
template <int G, int R, int U, class T, bool YG = false>
__device__ __forceinline__ void primalRowsFrom(const IterArgs<T>& p, int j0, int jend, const int (&b)[R],
                                               const int (&e)[R], int koff) {
    constexpr int slab = kBlock / G;
    const int lane = threadIdx.x % G;
    const ColPack<T>* __restrict__ cp = p.cp;
    const double* __restrict__ xcp = p.xc;
    const T* __restrict__ xip = p.xi;
    ColPack<T> q[R];
    double xc[R];
    T xi[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int j = j0 + r * slab;
        q[r] = ColPack<T>{T(0), T(0), T(0), T(0)};
        xc[r] = 0.0;
        xi[r] = T(0);
        if (j < jend && lane == 0) {
            q[r] = cp[j];
            xc[r] = xcp[j];
            xi[r] = xip[j];
        }
    }
    double s[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        if constexpr (YG)
            s[r] = rowDotU<G, U, double>(b[r], e[r], lane, p.at_idx, p.at_val, p.yg);
        else
            s[r] = rowDotU<G, U, double>(b[r], e[r], lane, p.at_idx, p.at_val, p.yc);
    }
    bool last = false;
    if (!active(p.st, precTag<T>(), koff, p.max_iter, p.polish_max_iter, last, p.N)) return;
#pragma unroll
    for (int r = 0; r < R; ++r) s[r] = groupSum<G>(s[r]);
    const double step = p.st->step, pw = p.st->pw;
    const int k = p.st->inner + koff;
    const double lam = static_cast<double>(k) / static_cast<double>(k + 1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int j = j0 + r * slab;
        if (lane != 0 || j >= jend) continue;
        primalUpdate<T>(p, j, q[r], xc[r], static_cast<double>(xi[r]), s[r], step, pw, lam, last);
    }
}

// primalRows handles the columns j0 + r * slab (r < R) below jend; the
// single-LP kernel covers [0, n), the batched kernel one tile of one LP.
template <int G, int R, int U, class T, bool YG = false>
__device__ __forceinline__ void primalRows(const IterArgs<T>& p, int j0, int jend, int koff) {
    int b[R], e[R];
    rowBounds<G, R>(p.at_ptr, j0, jend, b, e);
    primalRowsFrom<G, R, U, T, YG>(p, j0, jend, b, e, koff);
}

// Columns [begin, end) of A^T (the engine launches long and short columns
// separately when their lengths are far apart).
template <int G, int R, int U, class T, bool YG = false>
__global__ void __launch_bounds__(kBlock) primalStep(IterArgs<T> p, int koff, int begin, int end) {
    constexpr int slab = kBlock / G;
    primalRows<G, R, U, T, YG>(p, begin + static_cast<int>(blockIdx.x) * (slab * R) + static_cast<int>(threadIdx.x) / G, end,
                           koff);
}

// Fused A x_refl + dual proximal step (pdlp_kernels.cu:94-157), same structure.
template <int G, int R, int U, class T>
__device__ __forceinline__ void dualRowsFrom(const IterArgs<T>& p, int i0, int iend, const int (&b)[R],
                                             const int (&e)[R], int koff) {
    constexpr int slab = kBlock / G;
    const int lane = threadIdx.x % G;
    const RowPack<T>* __restrict__ rp = p.rp;
    const double* __restrict__ ycp = p.yc;
    const T* __restrict__ yip = p.yi;
    RowPack<T> q[R];
    double yc[R];
    T yi[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = i0 + r * slab;
        q[r] = RowPack<T>{T(0), T(0), T(0), T(0)};
        yc[r] = 0.0;
        yi[r] = T(0);
        if (i < iend && lane == 0) {
            q[r] = rp[i];
            yc[r] = ycp[i];
            yi[r] = yip[i];
        }
    }
    double s[R];
#pragma unroll
    for (int r = 0; r < R; ++r) s[r] = rowDotU<G, U, double>(b[r], e[r], lane, p.a_idx, p.a_val, p.xr);
    bool last = false;
    if (!active(p.st, precTag<T>(), koff, p.max_iter, p.polish_max_iter, last, p.N)) return;
#pragma unroll
    for (int r = 0; r < R; ++r) s[r] = groupSum<G>(s[r]);
    const double step = p.st->step, pw = p.st->pw;
    const int k = p.st->inner + koff;
    const double lam = static_cast<double>(k) / static_cast<double>(k + 1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = i0 + r * slab;
        if (lane != 0 || i >= iend) continue;
        dualUpdate<T>(p, i, q[r], yc[r], static_cast<double>(yi[r]), s[r], step, pw, lam, last);
    }
}

template <int G, int R, int U, class T>
__device__ __forceinline__ void dualRows(const IterArgs<T>& p, int i0, int iend, int koff) {
    int b[R], e[R];
    rowBounds<G, R>(p.a_ptr, i0, iend, b, e);
    dualRowsFrom<G, R, U, T>(p, i0, iend, b, e, koff);
}

template <int G, int R, int U, class T>
__global__ void __launch_bounds__(kBlock) dualStep(IterArgs<T> p, int koff, int begin, int end) {
    constexpr int slab = kBlock / G;
    dualRows<G, R, U, T>(p, begin + static_cast<int>(blockIdx.x) * (slab * R) + static_cast<int>(threadIdx.x) / G, end,
                         koff);
}

// ---- programmatic dependent launch ------------------------------------------
// Step kernels launched with programmatic stream serialization may start while
// the kernel before them finishes its last wave.  pdlWait() returns once every
// grid this one depends on has completed and its writes are visible; code
// before it may read only data that no kernel still running writes.
// pdlTrigger() lets the next such kernel be scheduled once every block of this
// one has called it.  Both are no-ops for a kernel launched the usual way.
__device__ __forceinline__ void pdlWait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdlTrigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---- sliced ELL (SELL-32) step ----------------------------------------------
// A matrix side stored as 32-row slices: entry k of the slice's row `lane` sits
// at hdr.x + k * 32 + lane, hdr.y is the slice's longest row, and shorter rows
// are padded with index 0 / value 0 (index 0 exists whenever the side has a
// column).  One thread owns one row, so a warp's load of its rows' k-th entries
// is one coalesced request.  Used by the single-LP engine for its short rows
// and by the packed batch for whole tiles.
constexpr int kSlice = 32;           // rows per slice (one warp)
constexpr int kSellU[] = {4, 8, 16};  // entries per thread per round of the variants
constexpr int kNumSell = 3;

// Loads of the matrix stream (indices and values, read once per step) that
// neither allocate in L1 nor stay in L2 ahead of other lines (evict-first L2
// policy), so L1 and L2 keep the gathered iterate vectors.
__device__ __forceinline__ unsigned long long evictFirstPolicy() {
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ int ldStream(const int* a, unsigned long long pol) {
    int v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ float ldStream(const float* a, unsigned long long pol) {
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ double ldStream(const double* a, unsigned long long pol) {
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}

// Dot product of this thread's row with x: entry k of the row sits at
// hdr.x + k * 32 + lane; U entries are loaded per round, then their U gathers,
// then the products are summed in entry order (so every U, either kind of
// load, and either source of a gathered value give the same bits).  ST: the
// index / value loads use the streaming hints above.  HOT: x[0, H) -- the
// other side's longest rows, which the device numbering puts first -- is also
// held in shared memory at xs, and gathers of those entries read it there
// instead of through L1 (whose tag stage serves one sector of a scattered
// gather per clock).  Entries past the row's end hold index 0 and value 0
// (index 0 always exists).
template <int U, class V, class X, bool ST = false, bool HOT = false>
__device__ __forceinline__ double sellDot(const int* __restrict__ idx, const V* __restrict__ val, int2 h, int lane,
                                          const X* __restrict__ x, const X* xs = nullptr, int H = 0) {
    const int* ip = idx + h.x + lane;
    const V* vp = val + h.x + lane;
    double acc = 0.0;
    unsigned long long pol = 0;
    if constexpr (ST) pol = evictFirstPolicy();
    for (int k0 = 0; k0 < h.y; k0 += U) {
        int c[U];
        V v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int k = k0 + u;
            const bool ok = k < h.y;
            if constexpr (ST) {
                c[u] = ok ? ldStream(ip + k * kSlice, pol) : 0;
                v[u] = ok ? ldStream(vp + k * kSlice, pol) : V(0);
            } else {
                c[u] = ok ? __ldg(ip + k * kSlice) : 0;
                v[u] = ok ? __ldg(vp + k * kSlice) : V(0);
            }
        }
        X g[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if constexpr (HOT)
                g[u] = c[u] < H ? xs[c[u]] : __ldg(x + c[u]);
            else
                g[u] = __ldg(x + c[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) acc += static_cast<double>(v[u]) * static_cast<double>(g[u]);
    }
    return acc;
}

template <int U, class T, bool ST = false, bool HOT = false, bool YG = false>
__device__ __forceinline__ void primalSellFrom(const IterArgs<T>& p, const int* idx, const T* val, int j, int2 h,
                                               int koff, const T* ys = nullptr, int H = 0) {
    const ColPack<T> q = p.cp[j];
    const double xc = p.xc[j];
    const double xi = static_cast<double>(p.xi[j]);
    double s;
    if constexpr (YG)
        s = sellDot<U, T, T, ST, HOT>(idx, val, h, static_cast<int>(threadIdx.x) & 31, p.yg, ys, H);
    else
        s = sellDot<U, T, double, ST>(idx, val, h, static_cast<int>(threadIdx.x) & 31, p.yc);
    bool last = false;
    if (!active(p.st, precTag<T>(), koff, p.max_iter, p.polish_max_iter, last, p.N)) return;
    const double step = p.st->step, pw = p.st->pw;
    const int k = p.st->inner + koff;
    const double lam = static_cast<double>(k) / static_cast<double>(k + 1);
    primalUpdate<T>(p, j, q, xc, xi, s, step, pw, lam, last);
}

template <int U, class T, bool ST = false, bool HOT = false>
__device__ __forceinline__ void dualSellFrom(const IterArgs<T>& p, const int* idx, const T* val, int i, int2 h,
                                             int koff, const T* xs = nullptr, int H = 0) {
    const RowPack<T> q = p.rp[i];
    const double yc = p.yc[i];
    const double yi = static_cast<double>(p.yi[i]);
    const double s = sellDot<U, T, T, ST, HOT>(idx, val, h, static_cast<int>(threadIdx.x) & 31, p.xr, xs, H);
    bool last = false;
    if (!active(p.st, precTag<T>(), koff, p.max_iter, p.polish_max_iter, last, p.N)) return;
    const double step = p.st->step, pw = p.st->pw;
    const int k = p.st->inner + koff;
    const double lam = static_cast<double>(k) / static_cast<double>(k + 1);
    dualUpdate<T>(p, i, q, yc, yi, s, step, pw, lam, last);
}

// ---- block reduction of NS slots with per-slot operators -------------------
template <int NS>
__device__ __forceinline__ void blockReduceSlots(double (&acc)[NS], const int (&ops)[NS], double* out) {
    __shared__ double red[NS][kWarps];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        double v = acc[s];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_xor_sync(0xffffffffu, v, off);
            v = ops[s] == OP_SUM ? v + o : (ops[s] == OP_MIN ? fmin(v, o) : fmax(v, o));
        }
        if ((threadIdx.x & 31) == 0) red[s][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < NS) {
        const int s = threadIdx.x;
        double v = red[s][0];
        for (int w = 1; w < kWarps; ++w)
            v = ops[s] == OP_SUM ? v + red[s][w] : (ops[s] == OP_MIN ? fmin(v, red[s][w]) : fmax(v, red[s][w]));
        out[s] = v;
    }
}

__device__ __forceinline__ double slotInit(int op) {
    return op == OP_SUM ? 0.0 : (op == OP_MIN ? CUDART_INF : -CUDART_INF);
}

// Row terms of the check for one row with (A x_hat)_i = ax: primal residual
// (pdlp.cpp:1106-1117), dual-objective row term (pdlp.cpp:1185-1199), dual
// movement, and the Farkas / primal-ray certificate terms of pdlp.cpp:119-284
// in scaled space.
__device__ __forceinline__ void accRowMetrics(double (&acc)[kRowSlots], const DevConst& dc, double ax, double rl,
                                              double ru, double r, double y, double yi, double axabs = 0.0) {
    const double cl = ax < rl ? rl : (ru < ax ? ru : ax);
    const double v = (ax - cl) / (dc.con_scale * r);
    acc[R_PRES_SQ] += v * v;
    const double nz = axabs / (dc.con_scale * r);
    acc[R_NOISE_SQ] += nz * nz;
    acc[R_PRES_MAX] = fmax(acc[R_PRES_MAX], fabs(v));
    const double dy = y - yi;
    const bool hl = isfinite(rl), hu = isfinite(ru);
    double yp = y;
    if (!hu) yp = fmin(yp, 0.0);
    if (!hl) yp = fmax(yp, 0.0);
    if (yp > 0.0 && hu)
        acc[R_DOBJ_ROW] -= yp * ru;
    else if (yp < 0.0 && hl)
        acc[R_DOBJ_ROW] -= yp * rl;
    acc[R_DDIST] += dy * dy;
    const double yo = y * r;
    acc[R_YNORM] += yo * yo;
    const double yq = dc.obj_sign * yo;
    if (hu && !hl) acc[R_MIN_LE] = fmin(acc[R_MIN_LE], yq);
    if (hl && !hu) acc[R_MAX_GE] = fmax(acc[R_MAX_GE], yq);
    const double ys = dc.obj_sign * y;
    if (rl == ru)
        acc[R_FARKAS_ROW] += ys * rl;
    else if (ys > 0.0 && hu)
        acc[R_FARKAS_ROW] += ys * ru;
    else if (ys < 0.0 && hl)
        acc[R_FARKAS_ROW] += ys * rl;
    const double axr = ax / r;
    if (hl && hu)
        acc[R_UB_TWO] = fmax(acc[R_UB_TWO], fabs(axr));
    else if (hu)
        acc[R_UB_LE] = fmax(acc[R_UB_LE], axr);
    else if (hl)
        acc[R_UB_GE] = fmin(acc[R_UB_GE], axr);
}

// Column terms of the check for one column with (A^T y_hat)_j = aty and
// (A^T (y_hat - y_init))_j = atdy: primal objective, projected dual residual
// (pdlp.cpp:1123-1145), dual-objective column term (pdlp.cpp:1170-1184), primal
// movement and interaction, certificate terms.  Bound activity is judged
// against the bounds the iterate precision T clamped to: an FP32 x_hat sitting
// on float(ub) < ub is at its bound, not interior.
template <class T>
__device__ __forceinline__ void accColMetrics(double (&acc)[kColSlots], const DevConst& dc, double xh, double xi,
                                              double c, double lb, double ub, double cs, double aty, double atdy,
                                              double atyabs = 0.0) {
    const double dx = xh - xi;
    const bool hl = isfinite(lb), hu = isfinite(ub);
    acc[C_POBJ] += c * xh;
    const double g = c + aty;
    const double lbT = static_cast<double>(static_cast<T>(lb));
    const double ubT = static_cast<double>(static_cast<T>(ub));
    // A fixed column (lb == ub) admits a reduced cost of either sign, so it adds
    // no dual residual.  (The reference tests the lower bound first,
    // pdlp.cpp:1134-1140, and counts a negative reduced cost of a fixed column,
    // which never vanishes: LPs with fixed columns whose reduced cost is negative
    // cannot reach its tolerance.  dc.ref_fixed = 1 restores that behaviour.)
    double dr;
    if (hl && hu && lb == ub && !dc.ref_fixed)
        dr = 0.0;
    else if (xh <= lbT + 1e-12 && hl)
        dr = fmin(g, 0.0);
    else if (xh >= ubT - 1e-12 && hu)
        dr = fmax(g, 0.0);
    else
        dr = g;
    const double d = dr / (dc.obj_scale * cs);
    acc[C_DRES_SQ] += d * d;
    const double nd = atyabs / (dc.obj_scale * cs);
    acc[C_NOISE_SQ] += nd * nd;
    acc[C_DRES_MAX] = fmax(acc[C_DRES_MAX], fabs(d));
    double gp = g;
    if (!hl) gp = fmin(gp, 0.0);
    if (!hu) gp = fmax(gp, 0.0);
    if (gp > 0.0 && hl)
        acc[C_DOBJ_COL] += gp * lb;
    else if (gp < 0.0 && hu)
        acc[C_DOBJ_COL] += gp * ub;
    acc[C_PDIST] += dx * dx;
    acc[C_INTER] += atdy * dx;
    const double xo = xh * cs;
    acc[C_XNORM] += xo * xo;
    if (hl) acc[C_MIN_XLB] = fmin(acc[C_MIN_XLB], xo);
    if (hu) acc[C_MAX_XUB] = fmax(acc[C_MAX_XUB], xo);
    const double g2 = dc.obj_sign * aty;
    const double gq = g2 / cs;
    if (hl) acc[C_MIN_GLB] = fmin(acc[C_MIN_GLB], gq);
    if (hu) acc[C_MAX_GUB] = fmax(acc[C_MAX_GUB], gq);
    if (g2 > 0.0 && hl)
        acc[C_COLSUP] += g2 * lb;
    else if (g2 < 0.0 && hu)
        acc[C_COLSUP] += g2 * ub;
}

// FP64 row pass of the check: A x_hat and all row metrics (pdlp_kernels.cu:280-371,
// pdlp.cpp:1106-1120, 1185-1199, certificates pdlp.cpp:119-284) over rows
// lo + k * stride ... below hi; the block's partial slots go to out.
template <int G, class T>
__device__ __forceinline__ void checkRowsRange(const CheckArgs<T>& p, const DevConst& dc, int lo, int hi, int stride,
                                               double* out) {
    int ops[kRowSlots];
    double acc[kRowSlots];
#pragma unroll
    for (int s = 0; s < kRowSlots; ++s) {
        ops[s] = rowSlotOp(s);
        acc[s] = slotInit(ops[s]);
    }
    const int lane = threadIdx.x % G;
    const bool adapt = dc.adaptive != 0;
    for (int base = lo; base < hi; base += stride) {
        const int i = base + threadIdx.x / G;
        const bool valid = i < hi;
        double ax = 0.0, axa = 0.0;
        if (valid) ax = rowDotAbs<G>(p.a_ptr[i], p.a_ptr[i + 1], lane, p.a_idx, p.a_val, p.xh, axa);
        ax = groupSum<G>(ax);
        axa = groupSum<G>(axa);
        if (valid && lane == 0) {
            accRowMetrics(acc, dc, ax, p.rl64[i], p.ru64[i], p.rs64[i], static_cast<double>(p.yh[i]),
                          static_cast<double>(p.yi[i]), axa);
            if (adapt) {
                const double d = ax - p.prev_ax[i];
                acc[R_ADAPT] += p.sig64[i] * d * d;
                p.prev_ax[i] = ax;
            }
        }
    }
    blockReduceSlots<kRowSlots>(acc, ops, out);
}

// Rows [begin, end), block partials from slot part0 on.
template <int G, class T>
__global__ void __launch_bounds__(kBlock) checkRows(CheckArgs<T> p, int begin, int end, int part0) {
    const DevState* st = p.st;
    if (st->done || st->prec != precTag<T>()) return;
    constexpr int per_block = kBlock / G;
    checkRowsRange<G, T>(p, *p.dc, begin + static_cast<int>(blockIdx.x) * per_block, end, gridDim.x * per_block,
                         p.part_rows + static_cast<size_t>(part0 + blockIdx.x) * kRowSlots);
}

// FP64 column pass: A^T y_hat and A^T (y_hat - y_init) in one sweep, column
// metrics (pdlp_kernels.cu:163-274, pdlp.cpp:1123-1184, certificates).
template <int G, class T>
__device__ __forceinline__ void checkColsRange(const CheckArgs<T>& p, const DevConst& dc, int lo, int hi, int stride,
                                               double* out) {
    int ops[kColSlots];
    double acc[kColSlots];
#pragma unroll
    for (int s = 0; s < kColSlots; ++s) {
        ops[s] = colSlotOp(s);
        acc[s] = slotInit(ops[s]);
    }
    const int lane = threadIdx.x % G;
    const bool adapt = dc.adaptive != 0;
    for (int base = lo; base < hi; base += stride) {
        const int j = base + threadIdx.x / G;
        const bool valid = j < hi;
        double aty = 0.0, atdy = 0.0, atya = 0.0;
        if (valid) rowDot2<G>(p.at_ptr[j], p.at_ptr[j + 1], lane, p.at_idx, p.at_val, p.yh, p.yi, aty, atdy, atya);
        aty = groupSum<G>(aty);
        atdy = groupSum<G>(atdy);
        atya = groupSum<G>(atya);
        if (valid && lane == 0) {
            const double xh = static_cast<double>(p.xh[j]);
            accColMetrics<T>(acc, dc, xh, static_cast<double>(p.xi[j]), p.c64[j], p.lb64[j], p.ub64[j], p.cs64[j],
                             aty, atdy, atya);
            if (adapt) {
                const double dd = xh - p.prev_xh[j];
                acc[C_ADAPT] += dd * dd / p.tau64[j];
                p.prev_xh[j] = xh;
            }
        }
    }
    blockReduceSlots<kColSlots>(acc, ops, out);
}

template <int G, class T>
__global__ void __launch_bounds__(kBlock) checkCols(CheckArgs<T> p, int begin, int end, int part0) {
    const DevState* st = p.st;
    if (st->done || st->prec != precTag<T>()) return;
    constexpr int per_block = kBlock / G;
    checkColsRange<G, T>(p, *p.dc, begin + static_cast<int>(blockIdx.x) * per_block, end, gridDim.x * per_block,
                         p.part_cols + static_cast<size_t>(part0 + blockIdx.x) * kColSlots);
}

// Restart copy x_init = x_cur = x_hat, y_init = y_cur = y_hat (pdlp_kernels.cu:377-405),
// executed only when the controller decided to restart, and skipped when `skip`
// (the Anderson step's verdict, or null) says the extrapolated point was written
// instead.
template <class T>
__global__ void __launch_bounds__(kBlock) restartCopy(const DevState* st, int n, int m, const T* xh,
                                                     const T* yh, T* xi, T* yi, double* xc, double* yc,
                                                     const int* skip, T* yg) {
    if (st->done || st->prec != precTag<T>() || !st->restart) return;
    if (skip != nullptr && *skip) return;
    for (int k = blockIdx.x * kBlock + threadIdx.x; k < (n > m ? n : m); k += gridDim.x * kBlock) {
        if (k < n) {
            const T v = xh[k];
            xi[k] = v;
            xc[k] = v;
        }
        if (k < m) {
            const T v = yh[k];
            yi[k] = v;
            yc[k] = v;
            if constexpr (sizeof(T) == 4) {
                if (yg != nullptr) yg[k] = v;
            }
        }
    }
}

// FP32 -> FP64 hand-over of the iterate set (mixed precision mode).
struct PromoteArgs {  // the current iterates are FP64 in both modes and need no copy
    const float *xi, *xh, *yi, *yh;
    double *xi64, *xh64, *yi64, *yh64;
    DevState* st;
    int n, m;
};
__global__ void __launch_bounds__(kBlock) promoteIterates(PromoteArgs a);

__global__ void controller(DevState* st, const DevConst* dc, const double* part_rows,
                           const double* part_cols, DevState* host_mirror);

// ---- power iteration on A^T A (pdlp.cpp:748-795, 1985-2041) -----------------
struct PowerState {
    double s2;    // sigma^2 = x . A^T A x
    double nrm;   // ||A^T A x||
    double resid; // ||A^T A x - s2 x||
    int iter;
    int done;
};
struct PowerArgs {
    double* x;
    double* y;
    double* xn;
    double* part;  // [nb][2]
    PowerState* ps;
    int m, n, max_iter, nb;
    double tol;
};
template <class V>
struct PowerMat {
    const int* a_ptr;
    const int* a_idx;
    const V* a_val;
    const int* at_ptr;
    const int* at_idx;
    const V* at_val;
};
template <int G, class V>
__global__ void __launch_bounds__(kBlock) powerA(PowerArgs a, PowerMat<V> mt, int begin, int end) {
    if (a.ps->done) return;
    const int t = blockIdx.x * kBlock + threadIdx.x;
    const int i = begin + t / G, lane = t % G;
    const bool valid = i < end;
    double s = 0.0;
    if (valid) s = rowDot<G, double>(mt.a_ptr[i], mt.a_ptr[i + 1], lane, mt.a_idx, mt.a_val, a.x);
    s = groupSum<G>(s);
    if (valid && lane == 0) a.y[i] = s;
}
template <int G, class V>
__global__ void __launch_bounds__(kBlock) powerAt(PowerArgs a, PowerMat<V> mt, int begin, int end, int part0) {
    if (a.ps->done) return;
    const int per_block = kBlock / G;
    const int lane = threadIdx.x % G;
    double acc[2] = {0.0, 0.0};
    for (int base = begin + static_cast<int>(blockIdx.x) * per_block; base < end; base += gridDim.x * per_block) {
        const int j = base + threadIdx.x / G;
        const bool valid = j < end;
        double s = 0.0;
        if (valid) s = rowDot<G, double>(mt.at_ptr[j], mt.at_ptr[j + 1], lane, mt.at_idx, mt.at_val, a.y);
        s = groupSum<G>(s);
        if (valid && lane == 0) {
            a.xn[j] = s;
            acc[0] += a.x[j] * s;
            acc[1] += s * s;
        }
    }
    const int ops[2] = {OP_SUM, OP_SUM};
    blockReduceSlots<2>(acc, ops, a.part + static_cast<size_t>(part0 + blockIdx.x) * 2);
}
__global__ void powerFinish1(PowerArgs a);
__global__ void __launch_bounds__(kBlock) powerNormalize(PowerArgs a);
__global__ void powerFinish2(PowerArgs a);

// Plain SpMV for the parity entry point pdlpx_csr_spmv (FP64 accumulation, like the step kernels).
template <int G, class T>
__global__ void __launch_bounds__(kBlock) spmvKernel(int rows, const int* ptr, const int* idx, const T* val,
                                                    const T* x, T* y) {
    const int t = blockIdx.x * kBlock + threadIdx.x;
    const int i = t / G, lane = t % G;
    const bool valid = i < rows;
    double s = 0;
    if (valid) s = rowDot<G, double>(ptr[i], ptr[i + 1], lane, idx, val, x);
    s = groupSum<G>(s);
    if (valid && lane == 0) y[i] = static_cast<T>(s);
}

}  // namespace pdlpx
