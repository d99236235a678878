// Anderson acceleration at restarts on the device (single-LP engine).
//
// Type-I safeguarded Anderson acceleration (Walker & Ni 2011; Zhang,
// O'Donoghue & Boyd 2020) as PdlpSolver applies it at every main-loop restart
// (AndersonAccelerator, pdlp.cpp:293-437; GPU path pdlp.cpp:2082-2093 and
// 2418-2456): the pdhg iterate z = [x; y] and its residual r = z - z_anchor
// go into a ring of `w` slots; the Gram matrix of the last d = min(count, w)
// residuals, Tikhonov-regularised by reg * trace / d, is Cholesky-solved
// against the ones vector, the weights are normalised to sum 1, and the
// extrapolated point sum_i alpha_i z_i -- x clamped to the scaled column
// bounds -- replaces the restart point when |sum_i alpha_i r_i| is below
// |r_latest|; otherwise the plain restart copy runs.
//
// Device form, five launches per restart cycle, all inside the cycle graph and
// all returning at entry unless the controller has just decided a main-loop
// restart:
//   aaStore<T>      store z, r in the ring slot; block partials of the new
//                   Gram row (r_new . r_j for every filled slot j)
//   aaSolve         fixed-order reduction of the partials into the ring Gram
//                   matrix; ordered Gram, Cholesky, weights (one thread: d is
//                   the window, a handful of entries)
//   aaExtrapolate   sum_i alpha_i z_i into a scratch vector; block partials of
//                   |sum_i alpha_i r_i|^2 and |r_latest|^2
//   aaDecide        accept iff the first is below the second
//   aaApply<T>      accepted: scratch point -> anchor and current iterates
// restartCopy skips its copy when the extrapolation was accepted.  The Gram
// entries of older slots are kept between restarts instead of recomputed (the
// residuals they come from do not change), so each restart reads the new
// residual against the w stored ones once.  Sums are block partials reduced in
// a fixed order, so the decision is deterministic run to run.
#pragma once

#include "kernels.cuh"

namespace pdlpx {

struct AaState {
    int count;     // residuals stored so far (ring position = count % w)
    int d;         // depth of the last extrapolation
    int tried;     // a weight vector was computed this restart
    int accepted;  // the safeguard accepted the extrapolated point this restart
};

struct AaArgs {
    double* X;     // [w][n + m] stored iterates (pdhg x; pdhg y)
    double* Rr;    // [w][n + m] stored residuals (pdhg - anchor)
    double* out;   // [n + m] extrapolated point
    double* part;  // [nb][max(w, 2)] block partials
    double* gram;  // [w][w] Gram matrix indexed by ring slot
    double* work;  // [2 w w + 2 w] ordered Gram / Cholesky factor / z / weights
    int* order;    // [w] ring slot of the i-th oldest residual in the last extrapolation
    AaState* as;
    const DevState* st;
    const double* lb;  // scaled column bounds (clamp of the extrapolated x)
    const double* ub;
    int n, m, w, nb;
    double reg;
};

__device__ __forceinline__ bool aaRestartNow(const DevState* st) {
    return !st->done && st->restart && st->phase == 0;
}

// Sum over the block of one value per thread; the result is valid in thread 0.
__device__ __forceinline__ double aaBlockSum(double v) {
    __shared__ double red[kWarps];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    const int warp = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kWarps; ++w) t += red[w];
    return t;
}

template <class T>
__global__ void __launch_bounds__(kBlock) aaStore(AaArgs a, const T* xh, const T* xi, const T* yh, const T* yi) {
    if (!aaRestartNow(a.st) || a.st->prec != precTag<T>()) return;
    const int n = a.n, dim = a.n + a.m, w = a.w;
    const int slot = a.as->count % w;
    const int filled = a.as->count < w ? a.as->count : w;  // slots holding a residual before this store
    double* Xs = a.X + static_cast<size_t>(slot) * dim;
    double* Rs = a.Rr + static_cast<size_t>(slot) * dim;
    const int stride = gridDim.x * kBlock;
    double acc = 0.0;
    for (int k = blockIdx.x * kBlock + threadIdx.x; k < dim; k += stride) {
        double v, r;
        if (k < n) {
            v = static_cast<double>(xh[k]);
            r = v - static_cast<double>(xi[k]);
        } else {
            v = static_cast<double>(yh[k - n]);
            r = v - static_cast<double>(yi[k - n]);
        }
        Xs[k] = v;
        Rs[k] = r;
        acc += r * r;
    }
    const int ldp = w > 2 ? w : 2;
    double t = aaBlockSum(acc);
    if (threadIdx.x == 0) a.part[static_cast<size_t>(blockIdx.x) * ldp + slot] = t;
    for (int j = 0; j < filled; ++j) {
        if (j == slot) continue;
        const double* Rj = a.Rr + static_cast<size_t>(j) * dim;
        acc = 0.0;
        // the same thread wrote Rs[k] above: no synchronisation needed to read it back
        for (int k = blockIdx.x * kBlock + threadIdx.x; k < dim; k += stride) acc += Rs[k] * Rj[k];
        t = aaBlockSum(acc);
        if (threadIdx.x == 0) a.part[static_cast<size_t>(blockIdx.x) * ldp + j] = t;
    }
}

// One warp: lanes reduce the partials of the new Gram row, lane 0 solves.
__global__ void aaSolve(AaArgs a) {
    AaState* as = a.as;
    if (!aaRestartNow(a.st)) {
        if (threadIdx.x == 0) {
            as->tried = 0;
            as->accepted = 0;
        }
        return;
    }
    const int w = a.w, ldp = w > 2 ? w : 2;
    const int slot = as->count % w;
    const int filled = as->count < w ? as->count : w;
    for (int j = threadIdx.x; j < w; j += blockDim.x) {
        if (j != slot && j >= filled) continue;
        double s = 0.0;
        for (int b = 0; b < a.nb; ++b) s += a.part[static_cast<size_t>(b) * ldp + j];
        a.gram[static_cast<size_t>(slot) * w + j] = s;
        a.gram[static_cast<size_t>(j) * w + slot] = s;
    }
    __syncwarp();
    if (threadIdx.x != 0) return;
    const int count = as->count + 1;
    as->count = count;
    as->accepted = 0;
    as->tried = 0;
    const int d = count < w ? count : w;
    as->d = d;
    if (d < 2) return;
    double* g = a.work;           // [d][d] ordered, regularised Gram
    double* L = a.work + w * w;   // [d][d] Cholesky factor
    double* z = L + w * w;        // [d]
    double* alpha = z + w;        // [d]
    for (int i = 0; i < d; ++i) a.order[i] = (count - d + i) % w;
    for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) g[i * d + j] = a.gram[static_cast<size_t>(a.order[i]) * w + a.order[j]];
    double trace = 0.0;
    for (int i = 0; i < d; ++i) trace += g[i * d + i];
    const double mu = a.reg * trace / static_cast<double>(d);
    for (int i = 0; i < d; ++i) g[i * d + i] += mu;
    for (int i = 0; i < d * d; ++i) L[i] = 0.0;
    for (int i = 0; i < d; ++i) {
        for (int j = 0; j <= i; ++j) {
            double s = g[i * d + j];
            for (int p = 0; p < j; ++p) s -= L[i * d + p] * L[j * d + p];
            if (i == j) {
                if (s <= 0.0) return;  // not positive definite: plain restart
                L[i * d + j] = sqrt(s);
            } else {
                L[i * d + j] = s / L[j * d + j];
            }
        }
    }
    for (int i = 0; i < d; ++i) {  // L z = 1
        double s = 1.0;
        for (int p = 0; p < i; ++p) s -= L[i * d + p] * z[p];
        z[i] = s / L[i * d + i];
    }
    for (int i = d - 1; i >= 0; --i) {  // L^T alpha = z
        double s = z[i];
        for (int p = i + 1; p < d; ++p) s -= L[p * d + i] * alpha[p];
        alpha[i] = s / L[i * d + i];
    }
    double sum = 0.0;
    for (int i = 0; i < d; ++i) sum += alpha[i];
    if (fabs(sum) < 1e-15) return;
    for (int i = 0; i < d; ++i) alpha[i] /= sum;
    as->tried = 1;
}

__global__ void __launch_bounds__(kBlock) aaExtrapolate(AaArgs a) {
    const AaState* as = a.as;
    if (!as->tried) return;
    const int dim = a.n + a.m, w = a.w, d = as->d;
    const double* alpha = a.work + 2 * w * w + w;
    const double* Rl = a.Rr + static_cast<size_t>(a.order[d - 1]) * dim;
    double acc_aa = 0.0, acc_last = 0.0;
    for (int k = blockIdx.x * kBlock + threadIdx.x; k < dim; k += gridDim.x * kBlock) {
        double z = 0.0, r = 0.0;
        for (int i = 0; i < d; ++i) {
            const size_t base = static_cast<size_t>(a.order[i]) * dim + k;
            z += alpha[i] * a.X[base];
            r += alpha[i] * a.Rr[base];
        }
        a.out[k] = z;
        acc_aa += r * r;
        const double rl = Rl[k];
        acc_last += rl * rl;
    }
    const int ldp = w > 2 ? w : 2;
    const double t0 = aaBlockSum(acc_aa);
    const double t1 = aaBlockSum(acc_last);
    if (threadIdx.x == 0) {
        a.part[static_cast<size_t>(blockIdx.x) * ldp + 0] = t0;
        a.part[static_cast<size_t>(blockIdx.x) * ldp + 1] = t1;
    }
}

__global__ void aaDecide(AaArgs a) {
    AaState* as = a.as;
    if (threadIdx.x != 0 || !as->tried) return;
    const int ldp = a.w > 2 ? a.w : 2;
    double s0 = 0.0, s1 = 0.0;
    for (int b = 0; b < a.nb; ++b) {
        s0 += a.part[static_cast<size_t>(b) * ldp + 0];
        s1 += a.part[static_cast<size_t>(b) * ldp + 1];
    }
    as->accepted = s0 < s1 ? 1 : 0;
}

// Accepted extrapolation: x (clamped to the scaled bounds) and y become both
// the anchor and the current iterate (pdlp.cpp:2437-2456).
template <class T>
__global__ void __launch_bounds__(kBlock) aaApply(AaArgs a, T* xi, T* yi, double* xc, double* yc, T* yg) {
    if (!a.as->accepted || a.st->prec != precTag<T>()) return;
    const int n = a.n, m = a.m;
    const int total = n > m ? n : m;
    for (int k = blockIdx.x * kBlock + threadIdx.x; k < total; k += gridDim.x * kBlock) {
        if (k < n) {
            const T v = static_cast<T>(fmin(fmax(a.out[k], a.lb[k]), a.ub[k]));
            xi[k] = v;
            xc[k] = static_cast<double>(v);
        }
        if (k < m) {
            const T v = static_cast<T>(a.out[n + k]);
            yi[k] = v;
            yc[k] = static_cast<double>(v);
            if constexpr (sizeof(T) == 4) {
                if (yg != nullptr) yg[k] = v;
            }
        }
    }
}

}  // namespace pdlpx
