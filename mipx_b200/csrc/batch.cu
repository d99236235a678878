// Batched PDLP: many independent LPs in one persistent launch of thread-block
// clusters (pdlpx_batch_solve).
//
// Each cluster of K CTAs pulls LPs from an atomic queue (largest first) and
// solves one LP completely before taking the next: the LP's columns and rows
// are split across the K CTAs, the primal and dual phases of every PDHG
// iteration are separated by hardware cluster barriers, and the power
// iteration, FP64 check pass, controller (restart / primal weight / polish /
// termination, the same controlStep as the single-LP graph) and FP32 -> FP64
// hand-over all run inside the kernel.  Every CTA of a cluster reads the same
// partials after a barrier and runs the controller on its own copy of the
// solver state, so all control decisions -- and therefore the barrier
// sequence -- are identical across the cluster by construction; there are no
// spin waits.  Vectors written by other CTAs during the kernel are read with
// L2-coherent loads (ld.global.cg); the matrix and per-row / per-column
// constants are read-only for the whole launch.
//
// An LP is solved by one cluster with the same code and reduction order
// whatever else is in the batch, so its result is bit-identical alone and in
// any mix (batch invariance).
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <thread>
#include <vector>

#include "control.cuh"
#include "engine.hpp"
#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace pdlpx {
namespace {

constexpr int kMaxCluster = 8;
constexpr int kSlots = kRowSlots + kColSlots;
constexpr int kPartStride = kSlots + 3;  // per CTA rank: check slots + 3 power-iteration slots

struct BatchLp {
    IterArgs<float> it32;
    IterArgs<double> it64;
    CheckArgs<float> ck32;
    CheckArgs<double> ck64;
    const float* a_v32;
    const float* at_v32;
    double* pi_x;
    double* pi_y;
    double* pi_xn;
    double* part;  // [kMaxCluster][kPartStride]
    DevState* st;  // initial state in, final state out
    const DevConst* dc;
    int m, n, gA, gAT, mixed, sv_max_iter;
    double sv_tol;
    // Slices: rank r owns rows [r*pr, (r+1)*pr) and columns [r*pc, (r+1)*pc) (clipped).
    int pr, pc;
    // Shared-memory residency: 1 when the FP32 phase runs from the cluster's
    // shared memory; capA / capAT = largest per-rank nonzero count of A / A^T.
    int smem, capA, capAT;
};

// Shared-memory image of one CTA's slice (identical offsets on every rank, so a
// remote address is the local address mapped to the owner's rank).
struct SLayout {
    int o_cp, o_rp, o_xc, o_yc, o_aptr, o_aidx, o_aval, o_atptr, o_atidx, o_atval, o_xi, o_xh, o_xr, o_yi, o_yh;
    int bytes;
};

__host__ __device__ inline int sAlign(int b) { return (b + 15) & ~15; }

__host__ __device__ inline SLayout smemLayout(int pr, int pc, int capA, int capAT) {
    SLayout L{};
    int o = 0;
    L.o_cp = o;
    o += sAlign(16 * pc);
    L.o_rp = o;
    o += sAlign(16 * pr);
    L.o_xc = o;
    o += sAlign(8 * pc);
    L.o_yc = o;
    o += sAlign(8 * pr);
    L.o_aptr = o;
    o += sAlign(4 * (pr + 1));
    L.o_aidx = o;
    o += sAlign(4 * capA);
    L.o_aval = o;
    o += sAlign(4 * capA);
    L.o_atptr = o;
    o += sAlign(4 * (pc + 1));
    L.o_atidx = o;
    o += sAlign(4 * capAT);
    L.o_atval = o;
    o += sAlign(4 * capAT);
    L.o_xi = o;
    o += sAlign(4 * pc);
    L.o_xh = o;
    o += sAlign(4 * pc);
    L.o_xr = o;
    o += sAlign(4 * pc);
    L.o_yi = o;
    o += sAlign(4 * pr);
    L.o_yh = o;
    o += sAlign(4 * pr);
    L.bytes = o;
    return L;
}

// Dynamic shared memory requested per CTA when some LP of the batch is resident.
constexpr int kSmemBudget = 220 * 1024;

template <class X>
__device__ __forceinline__ double ldc(const X* p) {
    return static_cast<double>(__ldcg(p));
}

// Row dot product with the gathered vector read through L2 (coherent across
// the cluster's SMs); matrix entries through the read-only path.
template <int G, int U, class V, class X>
__device__ __forceinline__ double rowDotC(int b, int e, int lane, const int* __restrict__ idx,
                                          const V* __restrict__ val, const X* x) {
    double s[U];
#pragma unroll
    for (int u = 0; u < U; ++u) s[u] = 0.0;
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
        for (int u = 0; u < U; ++u) s[u] += static_cast<double>(v[u]) * ldc(x + c[u]);
    }
    double t = s[0];
#pragma unroll
    for (int u = 1; u < U; ++u) t += s[u];
    return t;
}

// ---- PDHG phases over a slice [lo, hi) of columns / rows -------------------
// Trip counts are block-uniform (all threads step `base` together), so the
// width-G shuffles of groupSum always see their whole warp.
template <int G, class T>
__device__ void slicePrimal(const IterArgs<T>& p, int lo, int hi, double step, double pw, double lam, bool last) {
    const int lane = threadIdx.x % G;
    constexpr int per = kBlock / G;
    for (int base = lo; base < hi; base += per) {
        const int j = base + threadIdx.x / G;
        const bool valid = j < hi;
        double s = 0.0;
        if (valid) s = rowDotC<G, 4>(p.at_ptr[j], p.at_ptr[j + 1], lane, p.at_idx, p.at_val, p.yc);
        s = groupSum<G>(s);
        if (valid && lane == 0) {
            const ColPack<T> q = p.cp[j];
            const double xcd = p.xc[j], xid = p.xi[j];
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
    }
}

template <int G, class T>
__device__ void sliceDual(const IterArgs<T>& p, int lo, int hi, double step, double pw, double lam, bool last) {
    const int lane = threadIdx.x % G;
    constexpr int per = kBlock / G;
    for (int base = lo; base < hi; base += per) {
        const int i = base + threadIdx.x / G;
        const bool valid = i < hi;
        double s = 0.0;
        if (valid) s = rowDotC<G, 4>(p.a_ptr[i], p.a_ptr[i + 1], lane, p.a_idx, p.a_val, p.xr);
        s = groupSum<G>(s);
        if (valid && lane == 0) {
            const RowPack<T> q = p.rp[i];
            const double ycd = p.yc[i], yid = p.yi[i];
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
            p.yc[i] = lam * yr + (1.0 - lam) * yid;
            if (last) p.yh[i] = static_cast<T>(py);
        }
    }
}

// ---- FP64 check pass over a slice (same per-row / per-column terms as checkRows / checkCols)
template <int G, class T>
__device__ void sliceCheckRows(const CheckArgs<T>& p, const DevConst& dc, int lo, int hi, double (&acc)[kRowSlots]) {
    const int lane = threadIdx.x % G;
    constexpr int per = kBlock / G;
    for (int base = lo; base < hi; base += per) {
        const int i = base + threadIdx.x / G;
        const bool valid = i < hi;
        double ax = 0.0;
        if (valid) ax = rowDotC<G, 4>(p.a_ptr[i], p.a_ptr[i + 1], lane, p.a_idx, p.a_val, p.xh);
        ax = groupSum<G>(ax);
        if (valid && lane == 0)
            accRowMetrics(acc, dc, ax, p.rl64[i], p.ru64[i], p.rs64[i], static_cast<double>(p.yh[i]),
                          static_cast<double>(p.yi[i]));
    }
}

template <int G, class T>
__device__ void sliceCheckCols(const CheckArgs<T>& p, const DevConst& dc, int lo, int hi, double (&acc)[kColSlots]) {
    const int lane = threadIdx.x % G;
    constexpr int per = kBlock / G;
    for (int base = lo; base < hi; base += per) {
        const int j = base + threadIdx.x / G;
        const bool valid = j < hi;
        double aty = 0.0, atdy = 0.0;
        if (valid) {
            for (int k = p.at_ptr[j] + lane; k < p.at_ptr[j + 1]; k += G) {
                const int c = __ldg(p.at_idx + k);
                const double v = __ldg(p.at_val + k);
                const double yv = ldc(p.yh + c);
                aty += v * yv;
                atdy += v * (yv - ldc(p.yi + c));
            }
        }
        aty = groupSum<G>(aty);
        atdy = groupSum<G>(atdy);
        if (valid && lane == 0)
            accColMetrics<T>(acc, dc, static_cast<double>(p.xh[j]), static_cast<double>(p.xi[j]), p.c64[j], p.lb64[j],
                             p.ub64[j], p.cs64[j], aty, atdy);
    }
}

// ---- power iteration phases ------------------------------------------------
template <int G, class V>
__device__ void slicePowerRows(const int* ptr, const int* idx, const V* val, const double* x, double* y, int lo,
                               int hi) {
    const int lane = threadIdx.x % G;
    constexpr int per = kBlock / G;
    for (int base = lo; base < hi; base += per) {
        const int i = base + threadIdx.x / G;
        const bool valid = i < hi;
        double s = 0.0;
        if (valid) s = rowDotC<G, 4>(ptr[i], ptr[i + 1], lane, idx, val, x);
        s = groupSum<G>(s);
        if (valid && lane == 0) y[i] = s;
    }
}

template <int G, class V>
__device__ void slicePowerCols(const int* ptr, const int* idx, const V* val, const double* y, const double* x,
                               double* xn, int lo, int hi, double (&acc)[2]) {
    const int lane = threadIdx.x % G;
    constexpr int per = kBlock / G;
    for (int base = lo; base < hi; base += per) {
        const int j = base + threadIdx.x / G;
        const bool valid = j < hi;
        double s = 0.0;
        if (valid) s = rowDotC<G, 4>(ptr[j], ptr[j + 1], lane, idx, val, y);
        s = groupSum<G>(s);
        if (valid && lane == 0) {
            xn[j] = s;
            acc[0] += x[j] * s;
            acc[1] += s * s;
        }
    }
}

#define PDLPX_BATCH_G(GV, CALL)                       \
    switch (GV) {                                     \
        case 1: { constexpr int GG = 1; CALL; } break;   \
        case 2: { constexpr int GG = 2; CALL; } break;   \
        case 4: { constexpr int GG = 4; CALL; } break;   \
        case 8: { constexpr int GG = 8; CALL; } break;   \
        case 16: { constexpr int GG = 16; CALL; } break; \
        default: { constexpr int GG = 32; CALL; } break; \
    }

__device__ inline int batchGroup(int g) { return g > 32 ? 32 : g; }

// Spectral-norm estimate of one LP by the cluster (pdlp.cpp:748-795, FP64 vectors).
template <class V>
__device__ double clusterPower(const BatchLp& d, const int* a_ptr, const int* a_idx, const V* a_val,
                               const int* at_ptr, const int* at_idx, const V* at_val, int rank, int K,
                               cg::cluster_group& cl, int r0, int r1, int c0, int c1, double* sred) {
    const int gA = batchGroup(d.gA), gAT = batchGroup(d.gAT);
    double s2 = 1.0;
    for (int it = 0; it < d.sv_max_iter; ++it) {
        PDLPX_BATCH_G(gA, (slicePowerRows<GG, V>(a_ptr, a_idx, a_val, d.pi_x, d.pi_y, r0, r1)));
        cl.sync();
        double acc[2] = {0.0, 0.0};
        PDLPX_BATCH_G(gAT, (slicePowerCols<GG, V>(at_ptr, at_idx, at_val, d.pi_y, d.pi_x, d.pi_xn, c0, c1, acc)));
        const int ops2[2] = {OP_SUM, OP_SUM};
        blockReduceSlots<2>(acc, ops2, d.part + rank * kPartStride + kSlots);
        cl.sync();
        if (threadIdx.x == 0) {
            double a = 0.0, b = 0.0;
            for (int r = 0; r < K; ++r) {
                a += ldc(d.part + r * kPartStride + kSlots);
                b += ldc(d.part + r * kPartStride + kSlots + 1);
            }
            sred[0] = a;
            sred[1] = sqrt(b);
        }
        __syncthreads();
        s2 = sred[0];
        const double nrm = sred[1];
        double acc1[1] = {0.0};
        for (int j = c0 + threadIdx.x; j < c1; j += kBlock) {
            const double xn = d.pi_xn[j];
            const double dd = xn - s2 * d.pi_x[j];
            acc1[0] += dd * dd;
            if (nrm >= 1e-15) d.pi_x[j] = xn / nrm;
        }
        const int ops1[1] = {OP_SUM};
        blockReduceSlots<1>(acc1, ops1, d.part + rank * kPartStride + kSlots + 2);
        cl.sync();
        if (threadIdx.x == 0) {
            double rr = 0.0;
            for (int r = 0; r < K; ++r) rr += ldc(d.part + r * kPartStride + kSlots + 2);
            sred[2] = sqrt(rr);
        }
        __syncthreads();
        const double resid = sred[2];
        __syncthreads();
        if (nrm < 1e-15 || resid < d.sv_tol * fabs(s2)) break;
    }
    return s2;
}

// One restart cycle of one LP: N iterations, check, controller, restart copy, hand-over.
template <class T>
__device__ void clusterCycle(const BatchLp& d, const IterArgs<T>& it, const CheckArgs<T>& ck, int rank, int K,
                             cg::cluster_group& cl, DevState& sst, const DevConst& sdc, int r0, int r1, int c0,
                             int c1) {
    const int gA = batchGroup(d.gA), gAT = batchGroup(d.gAT);
    const int cur = sst.phase == 0 ? sst.total : sst.polish_count;
    const int lim = sst.phase == 0 ? sdc.max_iter : sdc.polish_max_iter;
    const int batch = min(sdc.N, lim - cur);
    const double step = sst.step, pw = sst.pw;
    const int inner = sst.inner;
    for (int k = 1; k <= batch; ++k) {
        const double lam = static_cast<double>(inner + k) / static_cast<double>(inner + k + 1);
        const bool last = k == batch;
        PDLPX_BATCH_G(gAT, (slicePrimal<GG, T>(it, c0, c1, step, pw, lam, last)));
        cl.sync();
        PDLPX_BATCH_G(gA, (sliceDual<GG, T>(it, r0, r1, step, pw, lam, last)));
        cl.sync();
    }
    int rops[kRowSlots], cops[kColSlots];
    double racc[kRowSlots], cacc[kColSlots];
#pragma unroll
    for (int s = 0; s < kRowSlots; ++s) {
        rops[s] = rowSlotOp(s);
        racc[s] = slotInit(rops[s]);
    }
#pragma unroll
    for (int s = 0; s < kColSlots; ++s) {
        cops[s] = colSlotOp(s);
        cacc[s] = slotInit(cops[s]);
    }
    PDLPX_BATCH_G(gA, (sliceCheckRows<GG, T>(ck, sdc, r0, r1, racc)));
    PDLPX_BATCH_G(gAT, (sliceCheckCols<GG, T>(ck, sdc, c0, c1, cacc)));
    blockReduceSlots<kRowSlots>(racc, rops, d.part + rank * kPartStride);
    blockReduceSlots<kColSlots>(cacc, cops, d.part + rank * kPartStride + kRowSlots);
    cl.sync();
    if (threadIdx.x == 0) {
        double rows[kRowSlots], cols[kColSlots];
        for (int s = 0; s < kRowSlots; ++s) {
            double v = slotInit(rops[s]);
            for (int r = 0; r < K; ++r) {
                const double w = ldc(d.part + r * kPartStride + s);
                v = rops[s] == OP_SUM ? v + w : (rops[s] == OP_MIN ? fmin(v, w) : fmax(v, w));
            }
            rows[s] = v;
        }
        for (int s = 0; s < kColSlots; ++s) {
            double v = slotInit(cops[s]);
            for (int r = 0; r < K; ++r) {
                const double w = ldc(d.part + r * kPartStride + kRowSlots + s);
                v = cops[s] == OP_SUM ? v + w : (cops[s] == OP_MIN ? fmin(v, w) : fmax(v, w));
            }
            cols[s] = v;
        }
        controlStep(sst, sdc, rows, cols);
    }
    __syncthreads();
    if (sst.restart) {
        for (int j = c0 + threadIdx.x; j < c1; j += kBlock) {
            const T v = it.xh[j];
            it.xi[j] = v;
            it.xc[j] = static_cast<double>(v);
        }
        for (int i = r0 + threadIdx.x; i < r1; i += kBlock) {
            const T v = it.yh[i];
            it.yi[i] = v;
            it.yc[i] = static_cast<double>(v);
        }
    }
    if (sizeof(T) == 4 && sst.promote && sst.prec == 0 && !sst.done) {
        for (int j = c0 + threadIdx.x; j < c1; j += kBlock) {
            d.it64.xi[j] = d.it32.xi[j];
            d.it64.xh[j] = d.it32.xh[j];
        }
        for (int i = r0 + threadIdx.x; i < r1; i += kBlock) {
            d.it64.yi[i] = d.it32.yi[i];
            d.it64.yh[i] = d.it32.yh[i];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            sst.prec = 1;
            sst.switch_total = sst.total;
        }
    }
    __syncthreads();
    cl.sync();  // restart / hand-over writes visible before the next cycle's gathers
}

// ---------------------------------------------------------------------------
// Shared-memory-resident FP32 phase.  The CTA's slice of A (its rows) and A^T
// (its columns) with FP32 values, its packed constants and its iterates live
// in its shared memory for the whole FP32 phase; an entry of A / A^T stores its
// column / row as (owner rank << 24 | index within the owner's slice), so the
// gathers of x_refl and y_cur read the owner's shared memory directly through
// distributed shared memory.  HBM is touched only by the FP64 check pass.
// ---------------------------------------------------------------------------
__device__ inline unsigned encodeOwner(int g, int per) {
    const int o = g / per;
    return (static_cast<unsigned>(o) << 24) | static_cast<unsigned>(g - o * per);
}

__device__ void smemLoad(const BatchLp& d, char* sm, const SLayout& L, int r0, int nr, int c0, int nc, int& a_off,
                         int& at_off) {
    const IterArgs<float>& it = d.it32;
    a_off = nr > 0 ? __ldg(it.a_ptr + r0) : 0;
    at_off = nc > 0 ? __ldg(it.at_ptr + c0) : 0;
    const int a_len = nr > 0 ? __ldg(it.a_ptr + r0 + nr) - a_off : 0;
    const int at_len = nc > 0 ? __ldg(it.at_ptr + c0 + nc) - at_off : 0;
    int* aptr = reinterpret_cast<int*>(sm + L.o_aptr);
    unsigned* aidx = reinterpret_cast<unsigned*>(sm + L.o_aidx);
    float* aval = reinterpret_cast<float*>(sm + L.o_aval);
    int* atptr = reinterpret_cast<int*>(sm + L.o_atptr);
    unsigned* atidx = reinterpret_cast<unsigned*>(sm + L.o_atidx);
    float* atval = reinterpret_cast<float*>(sm + L.o_atval);
    for (int i = threadIdx.x; i <= nr; i += kBlock) aptr[i] = nr > 0 ? __ldg(it.a_ptr + r0 + i) - a_off : 0;
    for (int j = threadIdx.x; j <= nc; j += kBlock) atptr[j] = nc > 0 ? __ldg(it.at_ptr + c0 + j) - at_off : 0;
    for (int k = threadIdx.x; k < a_len; k += kBlock) {
        aidx[k] = encodeOwner(__ldg(it.a_idx + a_off + k), d.pc);
        aval[k] = __ldg(d.a_v32 + a_off + k);
    }
    for (int k = threadIdx.x; k < at_len; k += kBlock) {
        atidx[k] = encodeOwner(__ldg(it.at_idx + at_off + k), d.pr);
        atval[k] = __ldg(d.at_v32 + at_off + k);
    }
    float4* cp = reinterpret_cast<float4*>(sm + L.o_cp);
    float4* rp = reinterpret_cast<float4*>(sm + L.o_rp);
    double* xc = reinterpret_cast<double*>(sm + L.o_xc);
    double* yc = reinterpret_cast<double*>(sm + L.o_yc);
    float* xi = reinterpret_cast<float*>(sm + L.o_xi);
    float* xh = reinterpret_cast<float*>(sm + L.o_xh);
    float* yi = reinterpret_cast<float*>(sm + L.o_yi);
    float* yh = reinterpret_cast<float*>(sm + L.o_yh);
    const float4* gcp = reinterpret_cast<const float4*>(it.cp);
    const float4* grp = reinterpret_cast<const float4*>(it.rp);
    // Iterates through L2 only: this SM must not keep L1 copies of lines that
    // other SMs write later in the solve.
    for (int j = threadIdx.x; j < nc; j += kBlock) {
        cp[j] = __ldg(gcp + c0 + j);
        xc[j] = __ldcg(it.xc + c0 + j);
        xi[j] = __ldcg(it.xi + c0 + j);
        xh[j] = __ldcg(it.xh + c0 + j);
    }
    for (int i = threadIdx.x; i < nr; i += kBlock) {
        rp[i] = __ldg(grp + r0 + i);
        yc[i] = __ldcg(it.yc + r0 + i);
        yi[i] = __ldcg(it.yi + r0 + i);
        yh[i] = __ldcg(it.yh + r0 + i);
    }
}

// Write the slice's iterates back to the global FP32 / FP64 arrays.
__device__ void smemStore(const BatchLp& d, char* sm, const SLayout& L, int r0, int nr, int c0, int nc) {
    const IterArgs<float>& it = d.it32;
    const double* xc = reinterpret_cast<const double*>(sm + L.o_xc);
    const double* yc = reinterpret_cast<const double*>(sm + L.o_yc);
    const float* xi = reinterpret_cast<const float*>(sm + L.o_xi);
    const float* xh = reinterpret_cast<const float*>(sm + L.o_xh);
    const float* yi = reinterpret_cast<const float*>(sm + L.o_yi);
    const float* yh = reinterpret_cast<const float*>(sm + L.o_yh);
    for (int j = threadIdx.x; j < nc; j += kBlock) {
        it.xc[c0 + j] = xc[j];
        it.xi[c0 + j] = xi[j];
        it.xh[c0 + j] = xh[j];
    }
    for (int i = threadIdx.x; i < nr; i += kBlock) {
        it.yc[r0 + i] = yc[i];
        it.yi[r0 + i] = yi[i];
        it.yh[r0 + i] = yh[i];
    }
}

template <int G>
__device__ void smemPrimal(char* sm, const SLayout& L, cg::cluster_group& cl, int nc, double step, double pw,
                           double lam, bool last) {
    const int* ptr = reinterpret_cast<const int*>(sm + L.o_atptr);
    const unsigned* idx = reinterpret_cast<const unsigned*>(sm + L.o_atidx);
    const float* val = reinterpret_cast<const float*>(sm + L.o_atval);
    const float4* cp = reinterpret_cast<const float4*>(sm + L.o_cp);
    double* xc = reinterpret_cast<double*>(sm + L.o_xc);
    const float* xi = reinterpret_cast<const float*>(sm + L.o_xi);
    float* xh = reinterpret_cast<float*>(sm + L.o_xh);
    float* xr = reinterpret_cast<float*>(sm + L.o_xr);
    double* yc_local = reinterpret_cast<double*>(sm + L.o_yc);
    const int lane = threadIdx.x % G;
    constexpr int per = kBlock / G;
    for (int base = 0; base < nc; base += per) {
        const int jl = base + threadIdx.x / G;
        const bool valid = jl < nc;
        double s0 = 0.0, s1 = 0.0;
        if (valid) {
            const int e = ptr[jl + 1];
            int k = ptr[jl] + lane;
            for (; k + G < e; k += 2 * G) {
                const unsigned w0 = idx[k], w1 = idx[k + G];
                const double v0 = cl.map_shared_rank(yc_local, w0 >> 24)[w0 & 0xFFFFFFu];
                const double v1 = cl.map_shared_rank(yc_local, w1 >> 24)[w1 & 0xFFFFFFu];
                s0 += static_cast<double>(val[k]) * v0;
                s1 += static_cast<double>(val[k + G]) * v1;
            }
            if (k < e) {
                const unsigned w = idx[k];
                s0 += static_cast<double>(val[k]) * cl.map_shared_rank(yc_local, w >> 24)[w & 0xFFFFFFu];
            }
        }
        double s = groupSum<G>(s0 + s1);
        if (valid && lane == 0) {
            const float4 q = cp[jl];  // c, lb, ub, tau_base
            const double xcd = xc[jl], xid = xi[jl];
            const double tau = step * static_cast<double>(q.w) / pw;
            double xv = xcd - tau * (static_cast<double>(q.x) + s);
            const double lb = q.y, ub = q.z;
            if (xv < lb) xv = lb;
            if (xv > ub) xv = ub;
            const double xrv = 2.0 * xv - xcd;
            xr[jl] = static_cast<float>(xrv);
            xc[jl] = lam * xrv + (1.0 - lam) * xid;
            if (last) xh[jl] = static_cast<float>(xv);
        }
    }
}

template <int G>
__device__ void smemDual(char* sm, const SLayout& L, cg::cluster_group& cl, int nr, double step, double pw,
                         double lam, bool last) {
    const int* ptr = reinterpret_cast<const int*>(sm + L.o_aptr);
    const unsigned* idx = reinterpret_cast<const unsigned*>(sm + L.o_aidx);
    const float* val = reinterpret_cast<const float*>(sm + L.o_aval);
    const float4* rp = reinterpret_cast<const float4*>(sm + L.o_rp);
    double* yc = reinterpret_cast<double*>(sm + L.o_yc);
    const float* yi = reinterpret_cast<const float*>(sm + L.o_yi);
    float* yh = reinterpret_cast<float*>(sm + L.o_yh);
    float* xr_local = reinterpret_cast<float*>(sm + L.o_xr);
    const int lane = threadIdx.x % G;
    constexpr int per = kBlock / G;
    for (int base = 0; base < nr; base += per) {
        const int il = base + threadIdx.x / G;
        const bool valid = il < nr;
        double s0 = 0.0, s1 = 0.0;
        if (valid) {
            const int e = ptr[il + 1];
            int k = ptr[il] + lane;
            for (; k + G < e; k += 2 * G) {
                const unsigned w0 = idx[k], w1 = idx[k + G];
                const float v0 = cl.map_shared_rank(xr_local, w0 >> 24)[w0 & 0xFFFFFFu];
                const float v1 = cl.map_shared_rank(xr_local, w1 >> 24)[w1 & 0xFFFFFFu];
                s0 += static_cast<double>(val[k]) * static_cast<double>(v0);
                s1 += static_cast<double>(val[k + G]) * static_cast<double>(v1);
            }
            if (k < e) {
                const unsigned w = idx[k];
                s0 += static_cast<double>(val[k]) *
                      static_cast<double>(cl.map_shared_rank(xr_local, w >> 24)[w & 0xFFFFFFu]);
            }
        }
        double s = groupSum<G>(s0 + s1);
        if (valid && lane == 0) {
            const float4 q = rp[il];  // sigma_base, rl, ru, type
            const double ycd = yc[il], yid = yi[il];
            const double sig = step * static_cast<double>(q.x) * pw;
            const double v = ycd + sig * s;
            const double rl = q.y, ru = q.z;
            const int type = static_cast<int>(q.w);
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
            yc[il] = lam * yr + (1.0 - lam) * yid;
            if (last) yh[il] = static_cast<float>(py);
        }
    }
}

template <int G>
__device__ void smemCheckRows(const BatchLp& d, char* sm, const SLayout& L, cg::cluster_group& cl, const DevConst& dc,
                              int r0, int nr, int a_off, double (&acc)[kRowSlots]) {
    const int* ptr = reinterpret_cast<const int*>(sm + L.o_aptr);
    const unsigned* idx = reinterpret_cast<const unsigned*>(sm + L.o_aidx);
    const float* xh_local = reinterpret_cast<const float*>(sm + L.o_xh);
    const float* yh = reinterpret_cast<const float*>(sm + L.o_yh);
    const float* yi = reinterpret_cast<const float*>(sm + L.o_yi);
    const double* val64 = d.ck32.a_val + a_off;
    const int lane = threadIdx.x % G;
    constexpr int per = kBlock / G;
    for (int base = 0; base < nr; base += per) {
        const int il = base + threadIdx.x / G;
        const bool valid = il < nr;
        double ax = 0.0;
        if (valid) {
            for (int k = ptr[il] + lane; k < ptr[il + 1]; k += G) {
                const unsigned w = idx[k];
                ax += __ldg(val64 + k) * static_cast<double>(cl.map_shared_rank(xh_local, w >> 24)[w & 0xFFFFFFu]);
            }
        }
        ax = groupSum<G>(ax);
        if (valid && lane == 0) {
            const int i = r0 + il;
            accRowMetrics(acc, dc, ax, d.ck32.rl64[i], d.ck32.ru64[i], d.ck32.rs64[i], static_cast<double>(yh[il]),
                          static_cast<double>(yi[il]));
        }
    }
}

template <int G>
__device__ void smemCheckCols(const BatchLp& d, char* sm, const SLayout& L, cg::cluster_group& cl, const DevConst& dc,
                              int c0, int nc, int at_off, double (&acc)[kColSlots]) {
    const int* ptr = reinterpret_cast<const int*>(sm + L.o_atptr);
    const unsigned* idx = reinterpret_cast<const unsigned*>(sm + L.o_atidx);
    const float* yh_local = reinterpret_cast<const float*>(sm + L.o_yh);
    const float* yi_local = reinterpret_cast<const float*>(sm + L.o_yi);
    const float* xh = reinterpret_cast<const float*>(sm + L.o_xh);
    const float* xi = reinterpret_cast<const float*>(sm + L.o_xi);
    const double* val64 = d.ck32.at_val + at_off;
    const int lane = threadIdx.x % G;
    constexpr int per = kBlock / G;
    for (int base = 0; base < nc; base += per) {
        const int jl = base + threadIdx.x / G;
        const bool valid = jl < nc;
        double aty = 0.0, atdy = 0.0;
        if (valid) {
            for (int k = ptr[jl] + lane; k < ptr[jl + 1]; k += G) {
                const unsigned w = idx[k];
                const double v = __ldg(val64 + k);
                const double yv = cl.map_shared_rank(yh_local, w >> 24)[w & 0xFFFFFFu];
                const double y0 = cl.map_shared_rank(yi_local, w >> 24)[w & 0xFFFFFFu];
                aty += v * yv;
                atdy += v * (yv - y0);
            }
        }
        aty = groupSum<G>(aty);
        atdy = groupSum<G>(atdy);
        if (valid && lane == 0) {
            const int j = c0 + jl;
            accColMetrics<float>(acc, dc, static_cast<double>(xh[jl]), static_cast<double>(xi[jl]), d.ck32.c64[j],
                                 d.ck32.lb64[j], d.ck32.ub64[j], d.ck32.cs64[j], aty, atdy);
        }
    }
}

// Combine the K ranks' partials (fixed order) and run the controller; every
// CTA does this on its own copy of the state and reaches the same result.
__device__ void clusterControl(const BatchLp& d, int K, DevState& sst, const DevConst& sdc) {
    if (threadIdx.x != 0) return;
    double rows[kRowSlots], cols[kColSlots];
    for (int s = 0; s < kRowSlots; ++s) {
        const int op = rowSlotOp(s);
        double v = slotInit(op);
        for (int r = 0; r < K; ++r) {
            const double w = ldc(d.part + r * kPartStride + s);
            v = op == OP_SUM ? v + w : (op == OP_MIN ? fmin(v, w) : fmax(v, w));
        }
        rows[s] = v;
    }
    for (int s = 0; s < kColSlots; ++s) {
        const int op = colSlotOp(s);
        double v = slotInit(op);
        for (int r = 0; r < K; ++r) {
            const double w = ldc(d.part + r * kPartStride + kRowSlots + s);
            v = op == OP_SUM ? v + w : (op == OP_MIN ? fmin(v, w) : fmax(v, w));
        }
        cols[s] = v;
    }
    controlStep(sst, sdc, rows, cols);
}

// FP32 phase of one LP from shared memory; returns when the LP is done or
// handed over to the FP64 (global memory) path.
__device__ void smemRun(const BatchLp& d, int rank, int K, cg::cluster_group& cl, DevState& sst, const DevConst& sdc,
                        char* sm, int r0, int nr, int c0, int nc) {
    const SLayout L = smemLayout(d.pr, d.pc, d.capA, d.capAT);
    const int gA = batchGroup(d.gA), gAT = batchGroup(d.gAT);
    int a_off = 0, at_off = 0;
    smemLoad(d, sm, L, r0, nr, c0, nc, a_off, at_off);
    __syncthreads();
    cl.sync();  // every slice resident before the first remote gather
    int rops[kRowSlots], cops[kColSlots];
#pragma unroll
    for (int s = 0; s < kRowSlots; ++s) rops[s] = rowSlotOp(s);
#pragma unroll
    for (int s = 0; s < kColSlots; ++s) cops[s] = colSlotOp(s);
    while (!sst.done && sst.prec == 0) {
        const int cur = sst.phase == 0 ? sst.total : sst.polish_count;
        const int lim = sst.phase == 0 ? sdc.max_iter : sdc.polish_max_iter;
        const int batch = min(sdc.N, lim - cur);
        const double step = sst.step, pw = sst.pw;
        const int inner = sst.inner;
        for (int k = 1; k <= batch; ++k) {
            const double lam = static_cast<double>(inner + k) / static_cast<double>(inner + k + 1);
            const bool last = k == batch;
            PDLPX_BATCH_G(gAT, (smemPrimal<GG>(sm, L, cl, nc, step, pw, lam, last)));
            cl.sync();
            PDLPX_BATCH_G(gA, (smemDual<GG>(sm, L, cl, nr, step, pw, lam, last)));
            cl.sync();
        }
        double racc[kRowSlots], cacc[kColSlots];
#pragma unroll
        for (int s = 0; s < kRowSlots; ++s) racc[s] = slotInit(rops[s]);
#pragma unroll
        for (int s = 0; s < kColSlots; ++s) cacc[s] = slotInit(cops[s]);
        PDLPX_BATCH_G(gA, (smemCheckRows<GG>(d, sm, L, cl, sdc, r0, nr, a_off, racc)));
        PDLPX_BATCH_G(gAT, (smemCheckCols<GG>(d, sm, L, cl, sdc, c0, nc, at_off, cacc)));
        blockReduceSlots<kRowSlots>(racc, rops, d.part + rank * kPartStride);
        blockReduceSlots<kColSlots>(cacc, cops, d.part + rank * kPartStride + kRowSlots);
        cl.sync();
        clusterControl(d, K, sst, sdc);
        __syncthreads();
        if (sst.restart) {
            double* xc = reinterpret_cast<double*>(sm + L.o_xc);
            double* yc = reinterpret_cast<double*>(sm + L.o_yc);
            float* xi = reinterpret_cast<float*>(sm + L.o_xi);
            const float* xh = reinterpret_cast<const float*>(sm + L.o_xh);
            float* yi = reinterpret_cast<float*>(sm + L.o_yi);
            const float* yh = reinterpret_cast<const float*>(sm + L.o_yh);
            for (int j = threadIdx.x; j < nc; j += kBlock) {
                xi[j] = xh[j];
                xc[j] = static_cast<double>(xh[j]);
            }
            for (int i = threadIdx.x; i < nr; i += kBlock) {
                yi[i] = yh[i];
                yc[i] = static_cast<double>(yh[i]);
            }
        }
        __syncthreads();
        if (sst.promote && !sst.done) {
            // hand-over: slice back to global memory, then FP32 -> FP64 copies
            smemStore(d, sm, L, r0, nr, c0, nc);
            __syncthreads();
            for (int j = c0 + threadIdx.x; j < c0 + nc; j += kBlock) {
                d.it64.xi[j] = d.it32.xi[j];
                d.it64.xh[j] = d.it32.xh[j];
            }
            for (int i = r0 + threadIdx.x; i < r0 + nr; i += kBlock) {
                d.it64.yi[i] = d.it32.yi[i];
                d.it64.yh[i] = d.it32.yh[i];
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                sst.prec = 1;
                sst.switch_total = sst.total;
            }
        }
        __syncthreads();
        cl.sync();
    }
    if (sst.done) smemStore(d, sm, L, r0, nr, c0, nc);
    __syncthreads();
    cl.sync();  // global copies complete before any later global-path gather
}

__device__ void clusterSolve(const BatchLp& d, int rank, int K, cg::cluster_group& cl, DevState& sst,
                             DevConst& sdc, double* sred, char* sm) {
    if (threadIdx.x == 0) {
        sst = *d.st;
        sdc = *d.dc;
    }
    __syncthreads();
    const int r0 = min(d.m, rank * d.pr), r1 = min(d.m, (rank + 1) * d.pr);
    const int c0 = min(d.n, rank * d.pc), c1 = min(d.n, (rank + 1) * d.pc);
    double s2 = 1.0;
    if (d.sv_max_iter > 0) {
        if (d.mixed)
            s2 = clusterPower<float>(d, d.it32.a_ptr, d.it32.a_idx, d.a_v32, d.it32.at_ptr, d.it32.at_idx, d.at_v32,
                                     rank, K, cl, r0, r1, c0, c1, sred);
        else
            s2 = clusterPower<double>(d, d.it64.a_ptr, d.it64.a_idx, d.it64.a_val, d.it64.at_ptr, d.it64.at_idx,
                                      d.it64.at_val, rank, K, cl, r0, r1, c0, c1, sred);
    }
    if (threadIdx.x == 0) {
        sst.step = 0.998 / sqrt(fmax(s2, 1e-12));
        sst.best_pw = sst.pw;
    }
    __syncthreads();
    cl.sync();
    if (d.smem && sst.prec == 0 && !sst.done) smemRun(d, rank, K, cl, sst, sdc, sm, r0, r1 - r0, c0, c1 - c0);
    while (!sst.done) {
        if (sst.prec == 0)
            clusterCycle<float>(d, d.it32, d.ck32, rank, K, cl, sst, sdc, r0, r1, c0, c1);
        else
            clusterCycle<double>(d, d.it64, d.ck64, rank, K, cl, sst, sdc, r0, r1, c0, c1);
    }
    if (rank == 0 && threadIdx.x == 0) *d.st = sst;
}

__global__ void __launch_bounds__(kBlock) batchSolveKernel(const BatchLp* lps, const int* order, int count,
                                                          int* queue) {
    cg::cluster_group cl = cg::this_cluster();
    const int K = static_cast<int>(cl.num_blocks());
    const int rank = static_cast<int>(cl.block_rank());
    extern __shared__ __align__(16) char s_dyn[];
    __shared__ int s_next;
    __shared__ DevState sst;
    __shared__ DevConst sdc;
    __shared__ double sred[4];
    while (true) {
        if (rank == 0 && threadIdx.x == 0) s_next = atomicAdd(queue, 1);
        cl.sync();
        const int q = *cl.map_shared_rank(&s_next, 0);
        cl.sync();  // every CTA has read the index before rank 0 takes the next one
        if (q >= count) break;
        clusterSolve(lps[order[q]], rank, K, cl, sst, sdc, sred, s_dyn);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct Item {
    const pdlpx_lp* in = nullptr;
    HostLp lp;
    ScaledLp sc;
    bool trivial = false;
    int gA = 1, gAT = 1;
    int pr = 1, pc = 1, capA = 0, capAT = 0, smem = 0, sbytes = 0;
    size_t off = 0, bytes = 0;
    // offsets within the item's region
    size_t o_aptr, o_aidx, o_atptr, o_atidx, o_av64, o_atv64, o_av32, o_atv32, o_cp32, o_rp32, o_cp64, o_rp64;
    size_t o_c, o_lb, o_ub, o_cs, o_tau, o_rl, o_ru, o_rs, o_sig;
    size_t o_x32[3], o_y32[2], o_x64[4], o_y64[3], o_pix, o_piy, o_pixn, o_part, o_st, o_dc;
};

size_t al256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

void layoutItem(Item& it, bool mixed) {
    const size_t m = it.lp.m, n = it.lp.n, nnz = it.sc.a.nnz();
    size_t o = 0;
    auto take = [&](size_t b) {
        const size_t at = o;
        o += al256(b);
        return at;
    };
    it.o_aptr = take(4 * (m + 1));
    it.o_aidx = take(4 * nnz);
    it.o_atptr = take(4 * (n + 1));
    it.o_atidx = take(4 * nnz);
    it.o_av64 = take(8 * nnz);
    it.o_atv64 = take(8 * nnz);
    it.o_av32 = mixed ? take(4 * nnz) : 0;
    it.o_atv32 = mixed ? take(4 * nnz) : 0;
    it.o_cp32 = mixed ? take(16 * n) : 0;
    it.o_rp32 = mixed ? take(16 * m) : 0;
    it.o_cp64 = take(32 * n);
    it.o_rp64 = take(32 * m);
    it.o_c = take(8 * n);
    it.o_lb = take(8 * n);
    it.o_ub = take(8 * n);
    it.o_cs = take(8 * n);
    it.o_tau = take(8 * n);
    it.o_rl = take(8 * m);
    it.o_ru = take(8 * m);
    it.o_rs = take(8 * m);
    it.o_sig = take(8 * m);
    for (auto& v : it.o_x32) v = mixed ? take(4 * n) : 0;
    for (auto& v : it.o_y32) v = mixed ? take(4 * m) : 0;
    for (auto& v : it.o_x64) v = take(8 * n);
    for (auto& v : it.o_y64) v = take(8 * m);
    it.o_pix = take(8 * n);
    it.o_piy = take(8 * m);
    it.o_pixn = take(8 * n);
    it.o_part = take(8 * kMaxCluster * kPartStride);
    it.o_st = take(sizeof(DevState));
    it.o_dc = take(sizeof(DevConst));
    it.bytes = o;
}

// Uniform slices of K ranks and whether the FP32 phase fits the cluster's
// shared memory (largest rank's slice image within the per-CTA budget).
void residency(Item& it, int K, bool mixed, bool allow) {
    const int m = it.lp.m, n = it.lp.n;
    it.pr = (m + K - 1) / K;
    it.pc = (n + K - 1) / K;
    const auto& ap = it.sc.a.ptr;
    const auto& atp = it.sc.at.ptr;
    it.capA = it.capAT = 0;
    for (int r = 0; r < K; ++r) {
        const int r0 = std::min(m, r * it.pr), r1 = std::min(m, (r + 1) * it.pr);
        const int c0 = std::min(n, r * it.pc), c1 = std::min(n, (r + 1) * it.pc);
        it.capA = std::max(it.capA, ap[r1] - ap[r0]);
        it.capAT = std::max(it.capAT, atp[c1] - atp[c0]);
    }
    const SLayout L = smemLayout(it.pr, it.pc, it.capA, it.capAT);
    it.sbytes = L.bytes;
    it.smem = allow && mixed && L.bytes <= kSmemBudget && it.pr < (1 << 24) && it.pc < (1 << 24) ? 1 : 0;
}

template <class T>
void putv(char* base, size_t off, const std::vector<T>& v) {
    if (!v.empty()) std::memcpy(base + off, v.data(), v.size() * sizeof(T));
}

// Fill an item's region of the host staging image (everything the kernel reads).
void stageItem(const Item& it, const pdlpx_options& o, bool mixed, char* img) {
    char* b = img + it.off;
    const ScaledLp& sc = it.sc;
    const int32_t m = it.lp.m, n = it.lp.n;
    putv(b, it.o_aptr, sc.a.ptr);
    putv(b, it.o_aidx, sc.a.idx);
    putv(b, it.o_atptr, sc.at.ptr);
    putv(b, it.o_atidx, sc.at.idx);
    putv(b, it.o_av64, sc.a.val);
    putv(b, it.o_atv64, sc.at.val);
    if (mixed) {
        putv(b, it.o_av32, std::vector<float>(sc.a.val.begin(), sc.a.val.end()));
        putv(b, it.o_atv32, std::vector<float>(sc.at.val.begin(), sc.at.val.end()));
        auto* cp = reinterpret_cast<ColPack<float>*>(b + it.o_cp32);
        for (int32_t j = 0; j < n; ++j)
            cp[j] = ColPack<float>{static_cast<float>(sc.c[j]), static_cast<float>(sc.cl[j]),
                                   static_cast<float>(sc.cu[j]), static_cast<float>(sc.tau[j])};
        auto* rp = reinterpret_cast<RowPack<float>*>(b + it.o_rp32);
        for (int32_t i = 0; i < m; ++i)
            rp[i] = RowPack<float>{static_cast<float>(sc.sigma[i]), static_cast<float>(sc.rl[i]),
                                   static_cast<float>(sc.ru[i]), static_cast<float>(sc.row_type[i])};
    }
    auto* cp64 = reinterpret_cast<ColPack<double>*>(b + it.o_cp64);
    for (int32_t j = 0; j < n; ++j) cp64[j] = ColPack<double>{sc.c[j], sc.cl[j], sc.cu[j], sc.tau[j]};
    auto* rp64 = reinterpret_cast<RowPack<double>*>(b + it.o_rp64);
    for (int32_t i = 0; i < m; ++i)
        rp64[i] = RowPack<double>{sc.sigma[i], sc.rl[i], sc.ru[i], static_cast<double>(sc.row_type[i])};
    putv(b, it.o_c, sc.c);
    putv(b, it.o_lb, sc.cl);
    putv(b, it.o_ub, sc.cu);
    putv(b, it.o_cs, sc.col_scale);
    putv(b, it.o_tau, sc.tau);
    putv(b, it.o_rl, sc.rl);
    putv(b, it.o_ru, sc.ru);
    putv(b, it.o_rs, sc.row_scale);
    putv(b, it.o_sig, sc.sigma);
    // initial iterates: zero or the warm start scaled like pdlp.cpp:915-930
    std::vector<double> wx(n, 0.0), wy(m, 0.0);
    if (it.in->warm_x != nullptr && it.in->warm_y != nullptr) {
        for (int32_t j = 0; j < n; ++j) wx[j] = it.in->warm_x[j] / sc.col_scale[j] * sc.con_scale;
        for (int32_t i = 0; i < m; ++i) wy[i] = it.in->warm_y[i] * sc.obj_scale / (sc.obj_sign * sc.row_scale[i]);
    }
    if (mixed) {
        std::vector<float> fx(wx.begin(), wx.end()), fy(wy.begin(), wy.end());
        for (int k = 0; k < 3; ++k) putv(b, it.o_x32[k], fx);
        for (int k = 0; k < 2; ++k) putv(b, it.o_y32[k], fy);
        putv(b, it.o_x64[0], std::vector<double>(fx.begin(), fx.end()));
        putv(b, it.o_y64[0], std::vector<double>(fy.begin(), fy.end()));
    } else {
        for (int k = 0; k < 4; ++k) putv(b, it.o_x64[k], wx);
        for (int k = 0; k < 3; ++k) putv(b, it.o_y64[k], wy);
    }
    // power-iteration start vector: mt19937(42) normals, normalised (pdlp.cpp:754-764)
    std::mt19937 rng(42);
    std::normal_distribution<double> dist(0.0, 1.0);
    std::vector<double> x0(n);
    for (auto& v : x0) v = dist(rng);
    double xn = 0.0;
    for (double v : x0) xn += v * v;
    xn = std::sqrt(xn);
    if (xn < 1e-15) xn = 1.0;
    for (auto& v : x0) v /= xn;
    putv(b, it.o_pix, x0);
    // state and constants
    DevConst dc{};
    dc.m = m;
    dc.n = n;
    dc.N = o.termination_eval_frequency;
    dc.max_iter = o.max_iter;
    dc.polish_max_iter = o.polish_max_iter;
    dc.linf = o.optimality_norm == PDLPX_NORM_LINF;
    dc.update_pw = o.update_primal_weight != 0;
    dc.enable_polish = o.enable_polishing != 0;
    dc.mixed = mixed;
    dc.fp64_switch = o.fp64_switch != 0;
    dc.adaptive = 0;
    dc.precond_refresh = o.preconditioner_refresh != 0;
    dc.stall_limit = 10;
    dc.primal_tol = o.primal_tol;
    dc.dual_tol = o.dual_tol;
    dc.opt_tol = o.optimality_tol;
    dc.polish_ptol = o.polish_primal_tol;
    dc.polish_dtol = o.polish_dual_tol;
    dc.kp = o.pid_kp;
    dc.ki = o.pid_ki;
    dc.kd = o.pid_kd;
    dc.ismooth = o.pid_i_smooth;
    dc.suff = o.restart_sufficient_decay;
    dc.nec = o.restart_necessary_decay;
    dc.art = o.restart_artificial_fraction;
    terminationNorms(it.lp, o.optimality_norm, dc.c_norm, dc.b_norm);
    dc.obj_sign = sc.obj_sign;
    dc.obj_scale = sc.obj_scale;
    dc.con_scale = sc.con_scale;
    dc.offset = it.lp.offset;
    dc.precond_ratio = o.preconditioner_refresh_ratio;
    dc.switch_score = 30.0;
    std::memcpy(b + it.o_dc, &dc, sizeof(dc));
    DevState st{};
    st.pw = o.primal_weight;
    st.prec = mixed ? 0 : 1;
    st.fpe0 = -1.0;
    st.last_fpe = std::numeric_limits<double>::infinity();
    st.best_pw = st.pw;
    st.best_score = std::numeric_limits<double>::infinity();
    st.best_kkt = std::numeric_limits<double>::infinity();
    st.precond_pw = sc.precond_pw;
    st.switch_total = -1;
    std::memcpy(b + it.o_st, &st, sizeof(st));
}

BatchLp descriptor(const Item& it, char* dbase, const pdlpx_options& o, bool mixed) {
    char* b = dbase + it.off;
    auto I = [&](size_t off) { return reinterpret_cast<int*>(b + off); };
    auto F = [&](size_t off) { return reinterpret_cast<float*>(b + off); };
    auto D = [&](size_t off) { return reinterpret_cast<double*>(b + off); };
    BatchLp d{};
    d.m = it.lp.m;
    d.n = it.lp.n;
    d.gA = it.gA;
    d.gAT = it.gAT;
    d.mixed = mixed;
    d.sv_max_iter = o.sv_max_iter;
    d.sv_tol = o.sv_tol;
    d.pr = it.pr;
    d.pc = it.pc;
    d.capA = it.capA;
    d.capAT = it.capAT;
    d.smem = it.smem;
    DevState* st = reinterpret_cast<DevState*>(b + it.o_st);
    auto fillIter = [&](auto& a, auto* av, auto* atv, auto* cp, auto* rp, auto* xi, auto* xr, auto* xh, auto* yi,
                        auto* yh) {
        a.at_ptr = I(it.o_atptr);
        a.at_idx = I(it.o_atidx);
        a.at_val = atv;
        a.a_ptr = I(it.o_aptr);
        a.a_idx = I(it.o_aidx);
        a.a_val = av;
        a.cp = cp;
        a.rp = rp;
        a.xc = D(it.o_x64[0]);
        a.xi = xi;
        a.xr = xr;
        a.xh = xh;
        a.yc = D(it.o_y64[0]);
        a.yi = yi;
        a.yh = yh;
        a.st = st;
        a.m = it.lp.m;
        a.n = it.lp.n;
        a.max_iter = o.max_iter;
        a.polish_max_iter = o.polish_max_iter;
        a.N = o.termination_eval_frequency;
    };
    fillIter(d.it64, D(it.o_av64), D(it.o_atv64), reinterpret_cast<ColPack<double>*>(b + it.o_cp64),
             reinterpret_cast<RowPack<double>*>(b + it.o_rp64), D(it.o_x64[1]), D(it.o_x64[2]), D(it.o_x64[3]),
             D(it.o_y64[1]), D(it.o_y64[2]));
    if (mixed)
        fillIter(d.it32, F(it.o_av32), F(it.o_atv32), reinterpret_cast<ColPack<float>*>(b + it.o_cp32),
                 reinterpret_cast<RowPack<float>*>(b + it.o_rp32), F(it.o_x32[0]), F(it.o_x32[1]), F(it.o_x32[2]),
                 F(it.o_y32[0]), F(it.o_y32[1]));
    auto fillCheck = [&](auto& c, const auto& itr) {
        c.a_ptr = I(it.o_aptr);
        c.a_idx = I(it.o_aidx);
        c.a_val = D(it.o_av64);
        c.at_ptr = I(it.o_atptr);
        c.at_idx = I(it.o_atidx);
        c.at_val = D(it.o_atv64);
        c.xh = itr.xh;
        c.xi = itr.xi;
        c.yh = itr.yh;
        c.yi = itr.yi;
        c.c64 = D(it.o_c);
        c.lb64 = D(it.o_lb);
        c.ub64 = D(it.o_ub);
        c.cs64 = D(it.o_cs);
        c.tau64 = D(it.o_tau);
        c.rl64 = D(it.o_rl);
        c.ru64 = D(it.o_ru);
        c.rs64 = D(it.o_rs);
        c.sig64 = D(it.o_sig);
        c.m = it.lp.m;
        c.n = it.lp.n;
        c.st = st;
    };
    fillCheck(d.ck64, d.it64);
    if (mixed) fillCheck(d.ck32, d.it32);
    d.a_v32 = mixed ? F(it.o_av32) : nullptr;
    d.at_v32 = mixed ? F(it.o_atv32) : nullptr;
    d.pi_x = D(it.o_pix);
    d.pi_y = D(it.o_piy);
    d.pi_xn = D(it.o_pixn);
    d.part = D(it.o_part);
    d.st = st;
    d.dc = reinterpret_cast<DevConst*>(b + it.o_dc);
    return d;
}

template <class F>
void parallelFor(int count, F&& f) {
    const int hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const int nt = std::min(hw, std::max(1, count));
    std::vector<std::thread> ts;
    std::atomic<int> next{0};
    for (int t = 0; t < nt; ++t)
        ts.emplace_back([&] {
            for (int k = next++; k < count; k = next++) f(k);
        });
    for (auto& t : ts) t.join();
}

#define PDLPX_BCK(call)                                                              \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            err = std::string(#call) + " failed: " + cudaGetErrorString(e_);         \
            return e_ == cudaErrorMemoryAllocation ? PDLPX_E_NOMEM : PDLPX_E_CUDA;   \
        }                                                                            \
    } while (0)

}  // namespace

int32_t batchSolve(int32_t count, const pdlpx_lp* lps, const pdlpx_options& o, pdlpx_result* results,
                   double* const* x_out, double* const* y_out, std::string& err) {
    const auto t0 = std::chrono::steady_clock::now();
    if (o.anderson_acceleration && o.anderson_window_size >= 2) {
        err = "anderson_acceleration is not available in the device engine";
        return PDLPX_E_INVALID;
    }
    if (o.adaptive_step) {
        err = "adaptive_step is not available in the batched solve";
        return PDLPX_E_INVALID;
    }
    if (o.termination_eval_frequency <= 0) {
        err = "termination_eval_frequency must be positive";
        return PDLPX_E_INVALID;
    }
    const bool mixed = o.precision != PDLPX_PREC_FP64;
    int K = o.batch_cluster > 0 ? o.batch_cluster : 4;
    K = std::max(1, std::min(K, kMaxCluster));
    std::vector<Item> items(count);
    std::vector<int32_t> codes(count, PDLPX_OK);
    parallelFor(count, [&](int k) {
        Item& it = items[k];
        it.in = &lps[k];
        const pdlpx_lp& in = lps[k];
        HostLp& lp = it.lp;
        lp.m = in.m;
        lp.n = in.n;
        lp.maximize = in.sense == PDLPX_MAXIMIZE;
        if (in.m < 0 || in.n < 0 || !canonicalCsr(in.m, in.n, in.nnz, in.row_ptr, in.col_idx, in.val, lp.a) ||
            (in.n > 0 && (in.obj == nullptr || in.col_lb == nullptr || in.col_ub == nullptr)) ||
            (in.m > 0 && (in.row_lb == nullptr || in.row_ub == nullptr))) {
            codes[k] = PDLPX_E_INVALID;
            return;
        }
        lp.obj.assign(in.obj, in.obj + in.n);
        lp.cl.assign(in.col_lb, in.col_lb + in.n);
        lp.cu.assign(in.col_ub, in.col_ub + in.n);
        lp.rl.assign(in.row_lb, in.row_lb + in.m);
        lp.ru.assign(in.row_ub, in.row_ub + in.m);
        lp.offset = in.obj_offset;
        buildScaled(lp, o, it.sc);
        it.trivial = lp.m == 0 || lp.n == 0;
        it.gA = std::min(32, pickGroup(it.sc.a.nnz(), lp.m));
        it.gAT = std::min(32, pickGroup(it.sc.a.nnz(), lp.n));
        if (!it.trivial) {
            layoutItem(it, mixed);
            residency(it, K, mixed, o.batch_resident != 0);
        }
    });
    for (int k = 0; k < count; ++k)
        if (codes[k] != PDLPX_OK) {
            err = "invalid LP at index " + std::to_string(k);
            return codes[k];
        }
    // Trivial LPs (no rows or no columns) are closed form, like pdlp.cpp:812-860, via the engine.
    std::vector<int> dev_items;
    size_t total = 0;
    for (int k = 0; k < count; ++k) {
        if (items[k].trivial) continue;
        items[k].off = total;
        total += items[k].bytes;
        dev_items.push_back(k);
    }
    for (int k = 0; k < count; ++k) {
        if (!items[k].trivial) continue;
        Engine e;
        e.setOptions(o);
        const pdlpx_lp& in = lps[k];
        int32_t rc = e.load(in.m, in.n, in.nnz, in.row_ptr, in.col_idx, in.val, in.obj, in.col_lb, in.col_ub,
                            in.row_lb, in.row_ub, in.sense, in.obj_offset);
        if (rc == PDLPX_OK) rc = e.solve(&results[k]);
        if (rc != PDLPX_OK) {
            err = e.last_error;
            return rc;
        }
        if (x_out && x_out[k] && !e.primal().empty()) std::memcpy(x_out[k], e.primal().data(), 8 * e.primal().size());
        if (y_out && y_out[k] && !e.dual().empty()) std::memcpy(y_out[k], e.dual().data(), 8 * e.dual().size());
    }
    const int nd = static_cast<int>(dev_items.size());
    if (nd == 0) return PDLPX_OK;

    int devcount = 0;
    if (cudaGetDeviceCount(&devcount) != cudaSuccess || devcount <= 0) {
        err = "no CUDA device visible";
        return PDLPX_E_NO_DEVICE;
    }
    PDLPX_BCK(cudaSetDevice((o.device >= 0 && o.device < devcount) ? o.device : 0));
    // Host image of the whole arena, filled in parallel, uploaded in one copy.
    std::vector<char> img(total);
    parallelFor(nd, [&](int q) { stageItem(items[dev_items[q]], o, mixed, img.data()); });
    char* dbase = nullptr;
    PDLPX_BCK(cudaMalloc(reinterpret_cast<void**>(&dbase), total));
    struct Free {
        void* p;
        ~Free() { cudaFree(p); }
    } guard_arena{dbase};
    cudaStream_t s = nullptr;
    PDLPX_BCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct SFree {
        cudaStream_t s;
        ~SFree() { cudaStreamDestroy(s); }
    } guard_stream{s};
    PDLPX_BCK(cudaMemcpyAsync(dbase, img.data(), total, cudaMemcpyHostToDevice, s));
    // Descriptors, order (largest first), queue.
    std::vector<BatchLp> desc(nd);
    for (int q = 0; q < nd; ++q) desc[q] = descriptor(items[dev_items[q]], dbase, o, mixed);
    std::vector<int> order(nd);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return items[dev_items[a]].sc.a.nnz() > items[dev_items[b]].sc.a.nnz();
    });
    const size_t meta = al256(sizeof(BatchLp) * nd) + al256(sizeof(int) * nd) + 256;
    char* dmeta = nullptr;
    PDLPX_BCK(cudaMalloc(reinterpret_cast<void**>(&dmeta), meta));
    struct Free guard_meta {
        dmeta
    };
    BatchLp* d_desc = reinterpret_cast<BatchLp*>(dmeta);
    int* d_order = reinterpret_cast<int*>(dmeta + al256(sizeof(BatchLp) * nd));
    int* d_queue = reinterpret_cast<int*>(dmeta + al256(sizeof(BatchLp) * nd) + al256(sizeof(int) * nd));
    PDLPX_BCK(cudaMemcpyAsync(d_desc, desc.data(), sizeof(BatchLp) * nd, cudaMemcpyHostToDevice, s));
    PDLPX_BCK(cudaMemcpyAsync(d_order, order.data(), sizeof(int) * nd, cudaMemcpyHostToDevice, s));
    PDLPX_BCK(cudaMemsetAsync(d_queue, 0, sizeof(int), s));

    // Launch: clusters of K CTAs, as many clusters as can be co-resident; the
    // dynamic shared memory is the largest resident slice image of the batch.
    int dyn = 0;
    for (int q = 0; q < nd; ++q) dyn = std::max(dyn, items[dev_items[q]].smem ? items[dev_items[q]].sbytes : 0);
    if (dyn > 0) PDLPX_BCK(cudaFuncSetAttribute(batchSolveKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kBlock, 1, 1);
    cfg.dynamicSmemBytes = static_cast<size_t>(dyn);
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(K, 1, 1);
    int max_clusters = 0;
    PDLPX_BCK(cudaOccupancyMaxActiveClusters(&max_clusters, batchSolveKernel, &cfg));
    const int nclusters = std::max(1, std::min(max_clusters, nd));
    cfg.gridDim = dim3(K * nclusters, 1, 1);
    cudaEvent_t e0, e1;
    PDLPX_BCK(cudaEventCreate(&e0));
    PDLPX_BCK(cudaEventCreate(&e1));
    PDLPX_BCK(cudaEventRecord(e0, s));
    PDLPX_BCK(cudaLaunchKernelEx(&cfg, batchSolveKernel, static_cast<const BatchLp*>(d_desc),
                                 static_cast<const int*>(d_order), nd, d_queue));
    PDLPX_BCK(cudaEventRecord(e1, s));
    PDLPX_BCK(cudaEventSynchronize(e1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PDLPX_BCK(cudaGetLastError());

    // Results.
    std::vector<DevState> fin(nd);
    std::vector<std::vector<double>> xs(nd), ys(nd);
    for (int q = 0; q < nd; ++q) {
        const Item& it = items[dev_items[q]];
        char* b = dbase + it.off;
        PDLPX_BCK(cudaMemcpyAsync(&fin[q], b + it.o_st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    }
    PDLPX_BCK(cudaStreamSynchronize(s));
    std::vector<std::vector<float>> fx(nd), fy(nd);
    for (int q = 0; q < nd; ++q) {
        const Item& it = items[dev_items[q]];
        char* b = dbase + it.off;
        const int32_t m = it.lp.m, n = it.lp.n;
        xs[q].resize(n);
        ys[q].resize(m);
        if (fin[q].prec == 0) {
            fx[q].resize(n);
            fy[q].resize(m);
            PDLPX_BCK(cudaMemcpyAsync(fx[q].data(), b + it.o_x32[2], 4 * static_cast<size_t>(n),
                                      cudaMemcpyDeviceToHost, s));
            PDLPX_BCK(cudaMemcpyAsync(fy[q].data(), b + it.o_y32[1], 4 * static_cast<size_t>(m),
                                      cudaMemcpyDeviceToHost, s));
        } else {
            PDLPX_BCK(cudaMemcpyAsync(xs[q].data(), b + it.o_x64[3], 8 * static_cast<size_t>(n),
                                      cudaMemcpyDeviceToHost, s));
            PDLPX_BCK(cudaMemcpyAsync(ys[q].data(), b + it.o_y64[2], 8 * static_cast<size_t>(m),
                                      cudaMemcpyDeviceToHost, s));
        }
    }
    PDLPX_BCK(cudaStreamSynchronize(s));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    parallelFor(nd, [&](int q) {
        const int k = dev_items[q];
        const Item& it = items[k];
        const DevState& f = fin[q];
        const int32_t m = it.lp.m, n = it.lp.n;
        if (f.prec == 0) {
            for (int32_t j = 0; j < n; ++j) xs[q][j] = fx[q][j];
            for (int32_t i = 0; i < m; ++i) ys[q][i] = fy[q][i];
        }
        const ScaledLp& sc = it.sc;
        pdlpx_result& r = results[k];
        std::memset(&r, 0, sizeof(r));
        int32_t status = f.done ? f.status : (f.converged ? PDLPX_STATUS_OPTIMAL : PDLPX_STATUS_ITER_LIMIT);
        std::vector<double> xo(n, 0.0), yo(m, 0.0);
        double obj = 0.0;
        if (status == PDLPX_STATUS_OPTIMAL) {
            const double ic = 1.0 / sc.con_scale, io = 1.0 / sc.obj_scale;
            double ov = it.lp.offset;
            for (int32_t j = 0; j < n; ++j) {
                double xj = xs[q][j] * sc.col_scale[j] * ic;
                if (std::isfinite(it.lp.cl[j])) xj = std::max(xj, it.lp.cl[j]);
                if (std::isfinite(it.lp.cu[j])) xj = std::min(xj, it.lp.cu[j]);
                xo[j] = xj;
                ov += it.lp.obj[j] * xj;
            }
            for (int32_t i = 0; i < m; ++i) yo[i] = sc.obj_sign * ys[q][i] * sc.row_scale[i] * io;
            obj = ov;
        } else if (status == PDLPX_STATUS_INFEASIBLE) {
            const double io = 1.0 / sc.obj_scale;
            for (int32_t i = 0; i < m; ++i) yo[i] = sc.obj_sign * ys[q][i] * sc.row_scale[i] * io;
        } else if (status == PDLPX_STATUS_UNBOUNDED) {
            const double ic = 1.0 / sc.con_scale;
            for (int32_t j = 0; j < n; ++j) xo[j] = xs[q][j] * sc.col_scale[j] * ic;
        }
        r.status = status;
        r.objective = obj;
        r.iterations = f.total;
        r.work_units = static_cast<double>(f.total) *
                       (4.0 * static_cast<double>(sc.a.nnz()) + 2.0 * static_cast<double>(m + n));
        r.rel_primal_resid = f.pterm;
        r.rel_dual_resid = f.dterm;
        r.rel_gap = f.gap;
        r.primal_objective = f.pobj;
        r.dual_objective = f.dobj;
        r.fp64_iterations = mixed ? (f.switch_total >= 0 ? f.total - f.switch_total : 0) : f.total;
        r.restarts = f.restarts;
        r.step_size = f.step;
        r.primal_weight = f.pw;
        r.solve_seconds = secs;
        r.device_seconds = ms * 1e-3;
        r.used_gpu = 1;
        r.kernel_launches = 1;
        if (x_out && x_out[k]) std::memcpy(x_out[k], xo.data(), 8 * static_cast<size_t>(n));
        if (y_out && y_out[k]) std::memcpy(y_out[k], yo.data(), 8 * static_cast<size_t>(m));
    });
    return PDLPX_OK;
}

}  // namespace pdlpx
