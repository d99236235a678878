// Host orchestration of the PDLP engine and the non-template kernels.
//
// Solve flow (PdlpSolver::solve / solveGpu, pdlp.cpp:801-869, 1739-2792):
//   1. trivial cases on the host exactly as the reference (n == 0, m == 0);
//   2. device image of the scaled LP (FP32 and FP64 matrix values, packed
//      per-row / per-column constants, iterates) in one arena;
//   3. power iteration for the step size, device-resident, graph chunks;
//   4. restart cycles: one CUDA graph = N fused iterations + FP64 check +
//      controller + conditional restart copy (+ FP32->FP64 hand-over);
//      the host only reads the 200-byte state after each cycle to stop;
//   5. unscale on the host (pdlp.cpp:2678-2712).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <thread>
#include <limits>
#include <random>

#include "engine.hpp"
#include "kernels.cuh"
#include "anderson.cuh"
#include "control.cuh"
#include "shapes.cuh"

namespace pdlpx {

#define PDLPX_CK(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            err = std::string(#call) + " failed: " + cudaGetErrorString(e_);             \
            return e_ == cudaErrorMemoryAllocation ? PDLPX_E_NOMEM : PDLPX_E_CUDA;       \
        }                                                                                \
    } while (0)

// ---------------------------------------------------------------------------
// Non-template kernels
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kBlock) promoteIterates(PromoteArgs a) {
    const DevState* st = a.st;
    if (st->done || st->prec != 0 || !st->promote) return;
    const int total = a.n > a.m ? a.n : a.m;
    for (int k = blockIdx.x * kBlock + threadIdx.x; k < total; k += gridDim.x * kBlock) {
        if (k < a.n) {
            a.xi64[k] = a.xi[k];
            a.xh64[k] = a.xh[k];
        }
        if (k < a.m) {
            a.yi64[k] = a.yi[k];
            a.yh64[k] = a.yh[k];
        }
    }
}

__global__ void finishPromote(DevState* st) {
    if (!st->done && st->prec == 0 && st->promote) {
        st->prec = 1;
        st->switch_total = st->total;
    }
}

__global__ void __launch_bounds__(kBlock) controller(DevState* st, const DevConst* dc, const double* part_rows,
                                                    const double* part_cols, int prec) {
    if (st->done || st->prec != prec) return;
    __shared__ double rows[kRowSlots];
    __shared__ double cols[kColSlots];
    int rops[kRowSlots], cops[kColSlots];
#pragma unroll
    for (int s = 0; s < kRowSlots; ++s) rops[s] = rowSlotOp(s);
#pragma unroll
    for (int s = 0; s < kColSlots; ++s) cops[s] = colSlotOp(s);
    reducePartials<kRowSlots>(part_rows, dc->nb_rows, rops, rows);
    __syncthreads();
    reducePartials<kColSlots>(part_cols, dc->nb_cols, cops, cols);
    __syncthreads();
    if (threadIdx.x == 0) {
        DevState s = *st;
        controlStep(s, *dc, rows, cols);
        *st = s;
    }
}

// ---- power iteration -------------------------------------------------------
__global__ void __launch_bounds__(kBlock) powerFinish1(PowerArgs a) {
    if (a.ps->done) return;
    __shared__ double out[2];
    const int ops[2] = {OP_SUM, OP_SUM};
    reducePartials<2>(a.part, a.nb, ops, out);
    __syncthreads();
    if (threadIdx.x == 0) {
        a.ps->s2 = out[0];
        a.ps->nrm = sqrt(out[1]);
    }
}

__global__ void __launch_bounds__(kBlock) powerNormalize(PowerArgs a) {
    if (a.ps->done) return;
    const double s2 = a.ps->s2, nrm = a.ps->nrm;
    double acc[1] = {0.0};
    for (int j = blockIdx.x * kBlock + threadIdx.x; j < a.n; j += gridDim.x * kBlock) {
        const double xn = a.xn[j];
        const double d = xn - s2 * a.x[j];
        acc[0] += d * d;
        if (nrm >= 1e-15) a.x[j] = xn / nrm;
    }
    const int ops[1] = {OP_SUM};
    blockReduceSlots<1>(acc, ops, a.part + static_cast<size_t>(blockIdx.x) * 2);
}

__global__ void __launch_bounds__(kBlock) powerFinish2(PowerArgs a) {
    if (a.ps->done) return;
    __shared__ double out[1];
    double acc[1] = {0.0};
    for (int b = threadIdx.x; b < a.nb; b += kBlock) acc[0] += a.part[static_cast<size_t>(b) * 2];
    const int ops[1] = {OP_SUM};
    blockReduceSlots<1>(acc, ops, out);
    __syncthreads();
    if (threadIdx.x == 0) {
        PowerState& p = *a.ps;
        p.resid = sqrt(out[0]);
        p.iter += 1;
        if (p.nrm < 1e-15 || p.resid < a.tol * fabs(p.s2) || p.iter >= a.max_iter) p.done = 1;
    }
}

// ---- sliced-ELL step launches ------------------------------------------------
// The short rows [begin, end) of a matrix side stored as sliced ELL (slice s of
// the range described by hdr[s]); one thread per row, the fused step of
// kernels.cuh.  FP32 dual kernels are compiled for 8 resident blocks (32
// registers), the occupancy at which the packed batch's sliced-ELL kernels
// measured fastest; the FP32 primal kernels, which spilled 16-40 bytes per
// thread at 32 registers, for 6 (40 registers); the FP64 kernels, whose
// values and gathers take register pairs, for 5 (48 registers: at 32 they
// spilled 130-400 bytes per thread).
template <class T, bool PRIMAL = false>
constexpr int sellMinBlocks() {
    return sizeof(T) == 8 ? 5 : (PRIMAL ? 6 : 8);
}

template <int U, class T, bool ST>
__global__ void __launch_bounds__(kBlock, sellMinBlocks<T, true>())
    primalSellStep(IterArgs<T> p, const int2* __restrict__ hdr, const int* __restrict__ idx,
                   const T* __restrict__ val, int koff, int begin, int end) {
    const int r = static_cast<int>(blockIdx.x) * kBlock + static_cast<int>(threadIdx.x);
    if (begin + r >= end) return;
    primalSellFrom<U, T, ST, false, true>(p, idx, val, begin + r, hdr[r / kSlice], koff);
}

template <int U, class T, bool ST>
__global__ void __launch_bounds__(kBlock, sellMinBlocks<T>())
    dualSellStep(IterArgs<T> p, const int2* __restrict__ hdr, const int* __restrict__ idx,
                 const T* __restrict__ val, int koff, int begin, int end) {
    const int r = static_cast<int>(blockIdx.x) * kBlock + static_cast<int>(threadIdx.x);
    const int2 h = hdr[min(r, end - begin - 1) / kSlice];
    // the primal step before this one writes the x_refl gathered here and
    // reads the y written here
    pdlWait();
    pdlTrigger();
    if (begin + r >= end) return;
    dualSellFrom<U, T, ST>(p, idx, val, begin + r, h, koff);
}

// ---- sliced-ELL steps with the hot prefix of the gathered vector in shared memory
// The device numbering puts each side's long rows first, so the entries of the
// vector a step gathers that belong to the other side's longest rows form a
// prefix [0, H).  On power-law LPs a short prefix takes a large share of the
// gathers (on the 500k x 2M power-law LP the 4,096 longest columns hold 18 %
// of the nonzeros).  Each block first copies the prefix into shared memory
// with 16-byte loads, then runs the same per-row step as the kernels above
// with those gathers served from shared memory (same arithmetic and order, so
// the same bits).  Off unless the option asks for it: on that LP the dual step
// measured 78.6 us without the prefix and 91.7 / 100 / 226 us with 64 / 128 /
// 192 KB of shared memory per SM for it (B200, FP32): the shared memory is
// carved out of the L1 that already caches the popular columns and holds the
// sectors of the loads in flight.  (Persistent blocks holding a 110 KB prefix
// measured ~100 us too.)

// xs[0, H) = x[0, H) by the whole block (x 16-byte aligned), then a barrier.
template <class X>
__device__ __forceinline__ void fillHot(X* xs, const X* x, int H) {
    const int nv = static_cast<int>((static_cast<int64_t>(H) * static_cast<int64_t>(sizeof(X))) / 16);
    const int4* src = reinterpret_cast<const int4*>(x);
    int4* dst = reinterpret_cast<int4*>(xs);
    const int step = static_cast<int>(blockDim.x);
    for (int k = static_cast<int>(threadIdx.x); k < nv; k += step) dst[k] = __ldg(src + k);
    for (int k = nv * static_cast<int>(16 / sizeof(X)) + static_cast<int>(threadIdx.x); k < H; k += step)
        xs[k] = x[k];
    __syncthreads();
}

template <int U, class T, bool ST>
__global__ void __launch_bounds__(kBlock, sellMinBlocks<T, true>())
    primalSellHot(IterArgs<T> p, const int2* __restrict__ hdr, const int* __restrict__ idx,
                  const T* __restrict__ val, int koff, int begin, int end, int H) {
    extern __shared__ int4 hot_smem[];
    T* ys = reinterpret_cast<T*>(hot_smem);
    fillHot(ys, p.yg, H);
    const int r = static_cast<int>(blockIdx.x) * kBlock + static_cast<int>(threadIdx.x);
    if (begin + r >= end) return;
    primalSellFrom<U, T, ST, true, true>(p, idx, val, begin + r, hdr[r / kSlice], koff, ys, H);
}

template <int U, class T, bool ST>
__global__ void __launch_bounds__(kBlock, sellMinBlocks<T>())
    dualSellHot(IterArgs<T> p, const int2* __restrict__ hdr, const int* __restrict__ idx,
                const T* __restrict__ val, int koff, int begin, int end, int H) {
    extern __shared__ int4 hot_smem[];
    T* xs = reinterpret_cast<T*>(hot_smem);
    fillHot(xs, p.xr, H);
    const int r = static_cast<int>(blockIdx.x) * kBlock + static_cast<int>(threadIdx.x);
    if (begin + r >= end) return;
    dualSellFrom<U, T, ST, true>(p, idx, val, begin + r, hdr[r / kSlice], koff, xs, H);
}

// ---- long columns of the primal step in row chunks (mixed mode) ------------
// Every long column's gathers of y are scattered over all of y, and a gather
// through L1 costs its tag stage one sector whatever its size.  Cut into row
// chunks of R rows (R * 4 bytes of shared memory), each (chunk, column group)
// tile copies its chunk of the FP32 y into shared memory with 16-byte loads
// and serves every gather of its columns from there; 4 lanes per column sum
// the column's entries in the chunk (lane-strided, then a fixed shuffle tree)
// into part[j * C + c].  A second launch sums the C partials of each column
// in chunk order and runs the column's Halpern primal step.  The matrix copy
// stores rows as 16-bit offsets into the chunk (6 bytes per entry).
struct LongTileArgs {
    const int* off;        // [c * nl + j] .. [c * nl + j + 1]: entries of column j in chunk c
    const int* gb;         // G + 1 column-group bounds
    const uint16_t* row;   // row - c * R
    const float* val;
    double* part;          // [j * C + c]
    int R, C, G, nl;
    int maxcols;           // most columns in one group
};
constexpr int kTileBlock = 1024;
constexpr int kTileLanes = 4;
constexpr int kTileMaxRows = 28672;          // 112 KB of FP32 y per block

// shared memory of a tile: the chunk of y, then its group's offsets
static size_t tileSmemBytes(int R, int maxcols) {
    return 4 * static_cast<size_t>(R) + ((4 * static_cast<size_t>(maxcols + 1) + 15) & ~static_cast<size_t>(15));
}

__global__ void __launch_bounds__(kTileBlock, 1) primalLongTiles(IterArgs<float> p, LongTileArgs t, int koff) {
    bool last = false;
    if (!active(p.st, precTag<float>(), koff, p.max_iter, p.polish_max_iter, last, p.N)) return;
    extern __shared__ int4 tile_smem[];
    float* ys = reinterpret_cast<float*>(tile_smem);
    int* so = reinterpret_cast<int*>(ys + t.R);  // the group's entry offsets in this chunk
    const int c = static_cast<int>(blockIdx.x) / t.G, g = static_cast<int>(blockIdx.x) % t.G;
    const int j0 = t.gb[g], ncol = t.gb[g + 1] - j0;
    const int* __restrict__ off = t.off + static_cast<size_t>(c) * t.nl + j0;
    for (int q = static_cast<int>(threadIdx.x); q <= ncol; q += kTileBlock) so[q] = __ldg(off + q);
    // the dual step before this one writes the y copied here
    pdlWait();
    pdlTrigger();
    const int r0 = c * t.R;
    fillHot(ys, p.yg + r0, min(t.R, p.m - r0));  // ends with the block barrier
    const int lane = static_cast<int>(threadIdx.x) % kTileLanes;
    const int grp = static_cast<int>(threadIdx.x) / kTileLanes;
    constexpr int groups = kTileBlock / kTileLanes;
    // the 4 lanes of a group take the same columns, so their shuffles name
    // only themselves (groups of one warp may run different column counts)
    const unsigned mask = 0xFu << ((threadIdx.x & 31u) & ~3u);
    const uint16_t* __restrict__ row = t.row;
    const float* __restrict__ val = t.val;
    // two columns per pass, so two independent load chains are in flight
    for (int q = grp; q < ncol; q += 2 * groups) {
        const int q1 = q + groups;
        const int b0 = so[q], n0 = so[q + 1] - b0;
        const int b1 = q1 < ncol ? so[q1] : 0, n1 = q1 < ncol ? so[q1 + 1] - b1 : 0;
        double s0 = 0.0, s1 = 0.0;
        const int nmax = max(n0, n1);
#pragma unroll 2
        for (int r = lane; r < nmax; r += kTileLanes) {
            if (r < n0) s0 += static_cast<double>(__ldg(val + b0 + r)) * static_cast<double>(ys[__ldg(row + b0 + r)]);
            if (r < n1) s1 += static_cast<double>(__ldg(val + b1 + r)) * static_cast<double>(ys[__ldg(row + b1 + r)]);
        }
        s0 += __shfl_xor_sync(mask, s0, 1);
        s0 += __shfl_xor_sync(mask, s0, 2);
        s1 += __shfl_xor_sync(mask, s1, 1);
        s1 += __shfl_xor_sync(mask, s1, 2);
        if (lane == 0) {
            t.part[static_cast<size_t>(j0 + q) * t.C + c] = s0;
            if (q1 < ncol) t.part[static_cast<size_t>(j0 + q1) * t.C + c] = s1;
        }
    }
}

// Long column j: the sum of its chunk partials in chunk order, then its primal step.
__device__ __forceinline__ void longFinishColumn(const IterArgs<float>& p, const LongTileArgs& t, int j, int koff) {
    if (j >= t.nl) return;
    const ColPack<float> q = p.cp[j];
    const double xc = p.xc[j];
    const double xi = static_cast<double>(p.xi[j]);
    const double* __restrict__ pj = t.part + static_cast<size_t>(j) * t.C;
    double s = 0.0;
    for (int c = 0; c < t.C; ++c) s += pj[c];
    bool last = false;
    if (!active(p.st, precTag<float>(), koff, p.max_iter, p.polish_max_iter, last, p.N)) return;
    const double step = p.st->step, pw = p.st->pw;
    const int k = p.st->inner + koff;
    const double lam = static_cast<double>(k) / static_cast<double>(k + 1);
    primalUpdate<float>(p, j, q, xc, xi, s, step, pw, lam, last);
}

__global__ void __launch_bounds__(kBlock) primalLongFinish(IterArgs<float> p, LongTileArgs t, int koff) {
    longFinishColumn(p, t, static_cast<int>(blockIdx.x) * kBlock + static_cast<int>(threadIdx.x), koff);
}

// The finish of the long columns and the sliced-ELL step of the short ones in
// one launch: blocks [0, finish_blocks) finish long columns (first, so they
// overlap the short columns instead of trailing them), the rest run
// primalSellStep's work.  Same per-thread work as the two launches.
template <int U, bool ST>
__global__ void __launch_bounds__(kBlock, sellMinBlocks<float, true>())
    primalSellFinish(IterArgs<float> p, const int2* __restrict__ hdr, const int* __restrict__ idx,
                     const float* __restrict__ val, int koff, int begin, int end, LongTileArgs t, int finish_blocks) {
    const int b = static_cast<int>(blockIdx.x);
    // the tile launch before this one writes the partials the finish blocks
    // read; the short columns read only what earlier kernels wrote
    pdlTrigger();
    if (b < finish_blocks) {
        pdlWait();
        longFinishColumn(p, t, b * kBlock + static_cast<int>(threadIdx.x), koff);
        return;
    }
    const int r = (b - finish_blocks) * kBlock + static_cast<int>(threadIdx.x);
    if (begin + r >= end) return;
    primalSellFrom<U, float, ST, false, true>(p, idx, val, begin + r, hdr[r / kSlice], koff);
}

// ---- power iteration over the sliced-ELL sides --------------------------------
// The short rows of A (y = A x) and of A^T (x_n = A^T y, with the block
// partials of x . x_n and x_n . x_n) in the step kernels' layout: one thread
// per row, its entries summed in order in FP64, 8 per round.  On the
// 500k x 2M power-law LP the CSR A^T launch (2 lanes per column) took 3.3x the
// primal step's sliced-ELL time over the same columns.
template <class V>
__global__ void __launch_bounds__(kBlock) powerASell(PowerArgs a, const int2* __restrict__ hdr,
                                                    const int* __restrict__ idx, const V* __restrict__ val, int begin,
                                                    int end) {
    if (a.ps->done) return;
    const int r = static_cast<int>(blockIdx.x) * kBlock + static_cast<int>(threadIdx.x);
    if (begin + r >= end) return;
    a.y[begin + r] = sellDot<8, V, double>(idx, val, hdr[r / kSlice], static_cast<int>(threadIdx.x) & 31, a.x);
}

template <class V>
__global__ void __launch_bounds__(kBlock) powerAtSell(PowerArgs a, const int2* __restrict__ hdr,
                                                     const int* __restrict__ idx, const V* __restrict__ val, int begin,
                                                     int end, int part0) {
    if (a.ps->done) return;
    double acc[2] = {0.0, 0.0};
    const int rows = end - begin;
    // the stride is a multiple of 32, so a thread keeps its lane of every slice
    for (int r = static_cast<int>(blockIdx.x) * kBlock + static_cast<int>(threadIdx.x); r < rows;
         r += static_cast<int>(gridDim.x) * kBlock) {
        const int j = begin + r;
        const double s = sellDot<8, V, double>(idx, val, hdr[r / kSlice], static_cast<int>(threadIdx.x) & 31, a.y);
        a.xn[j] = s;
        acc[0] += a.x[j] * s;
        acc[1] += s * s;
    }
    const int ops[2] = {OP_SUM, OP_SUM};
    blockReduceSlots<2>(acc, ops, a.part + static_cast<size_t>(part0 + blockIdx.x) * 2);
}

// Sliced-ELL shapes of the single-LP engine: kNumShapes + k for k < kEngSell,
// U = kSellU[k % kNumSell], streaming loads for k >= kNumSell.
constexpr int kEngSell = 2 * kNumSell;
#define PDLPX_ENG_SELL_SWITCH(S, CALL)                                              \
    switch (S - kNumShapes) {                                                       \
        case 0: { constexpr int UU = kSellU[0]; constexpr bool SS = false; CALL; } break; \
        case 1: { constexpr int UU = kSellU[1]; constexpr bool SS = false; CALL; } break; \
        case 2: { constexpr int UU = kSellU[2]; constexpr bool SS = false; CALL; } break; \
        case 3: { constexpr int UU = kSellU[0]; constexpr bool SS = true; CALL; } break;  \
        case 4: { constexpr int UU = kSellU[1]; constexpr bool SS = true; CALL; } break;  \
        default: { constexpr int UU = kSellU[2]; constexpr bool SS = true; CALL; } break; \
    }

static int gridFor(int64_t rows, int G) {
    const int64_t threads = rows * G;
    return static_cast<int>(std::max<int64_t>(1, (threads + kBlock - 1) / kBlock));
}

int32_t pickGroup(int64_t nnz, int32_t rows) {
    if (rows <= 0) return 1;
    const double mean = static_cast<double>(nnz) / rows;
    if (mean <= 3) return 1;
    if (mean <= 6) return 2;
    if (mean <= 12) return 4;
    if (mean <= 24) return 8;
    if (mean <= 48) return 16;
    if (mean <= 128) return 32;
    if (mean <= 384) return 64;
    if (mean <= 768) return 128;
    return 256;
}

// ---------------------------------------------------------------------------
// Device image
// ---------------------------------------------------------------------------
struct DeviceLp {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    int m = 0, n = 0, nnz = 0;
    bool mixed = true;
    int gA = 1, gAT = 1;        // lanes per row of the check / power kernels
    int shapeP = 0, shapeD = 0;  // step kernel shapes (kShapes index): primal (A^T), dual (A)
    bool tuned = false;
    int nb_rows = 1, nb_cols = 1, nb_pi = 1;  // check / power partial blocks (all launches)
    // Rows of A (nlD) and of A^T (nlP) far longer than the rest come first in
    // the device numbering and get their own launches: lane counts gLA / gLAT,
    // step shapes shapeLD / shapeLP; the other rows use gA / gAT, shapeD / shapeP.
    int nlD = 0, nlP = 0, gLA = 1, gLAT = 1, shapeLD = 0, shapeLP = 0;
    int64_t zlD = 0, zlP = 0;  // entries of the long rows
    // hot prefixes: the primal step's gathers of y[0, hotP) and the dual step's
    // of x[0, hotD) are served from shared memory (0: off); the launch caps
    // them at what one block's shared memory holds
    int32_t hotP = 0, hotD = 0;
    int hot_smem_sm = 0, hot_smem_block = 0;  // shared memory per SM / per block (opt-in)
    int hot_bytes_sm = 0;                      // shared memory per SM given to the hot prefix
    // long columns in row chunks for the mixed-mode primal step (0 chunks: the
    // CSR launch runs instead); see buildLongTiles
    int lt_R = 0, lt_C = 0, lt_G = 0, lt_maxcols = 0;
    int32_t *lt_off = nullptr, *lt_gb = nullptr;
    uint16_t* lt_row = nullptr;
    float* lt_val = nullptr;
    double* lt_part = nullptr;
    LongTileArgs tiles() const {
        return LongTileArgs{lt_off, lt_gb, lt_row, lt_val, lt_part, lt_R, lt_C, lt_G, nlP, lt_maxcols};
    }
    int nb_rows_s = 1, nb_cols_s = 1, nb_pi_s = 1;  // partial blocks of the short-row launches
    std::vector<int32_t> rpos, cpos;  // original row / column -> device position (empty: identity)
    // Sides stored as sliced ELL (shapeP / shapeD >= kNumShapes): their short
    // rows [nl, rows) in 32-row slices; the CSR arrays stay for the long rows,
    // the check pass and the power iteration.
    int2* sp_hdr = nullptr;  // A^T short rows (primal step)
    int* sp_idx = nullptr;
    float* sp_v32 = nullptr;
    double* sp_v64 = nullptr;
    int2* sd_hdr = nullptr;  // A short rows (dual step)
    int* sd_idx = nullptr;
    float* sd_v32 = nullptr;
    double* sd_v64 = nullptr;
    // CUDA events recorded inside the cycle graphs around the primal and dual
    // step of iteration kev_iter of every cycle: [FP32 / FP64 graph][3]
    cudaEvent_t kev[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    int kev_iter = 1;

    int *a_ptr = nullptr, *a_idx = nullptr, *at_ptr = nullptr, *at_idx = nullptr;
    float *a_v32 = nullptr, *at_v32 = nullptr;
    double *a_v64 = nullptr, *at_v64 = nullptr;
    ColPack<float>* cp32 = nullptr;
    RowPack<float>* rp32 = nullptr;
    ColPack<double>* cp64 = nullptr;
    RowPack<double>* rp64 = nullptr;
    double *c64 = nullptr, *lb64 = nullptr, *ub64 = nullptr, *cs64 = nullptr, *tau64 = nullptr;
    double *rl64 = nullptr, *ru64 = nullptr, *rs64 = nullptr, *sig64 = nullptr;
    float *xi32 = nullptr, *xr32 = nullptr, *xh32 = nullptr;  // current x / y are always FP64
    float *yi32 = nullptr, *yh32 = nullptr;
    double *xc64 = nullptr, *xi64 = nullptr, *xr64 = nullptr, *xh64 = nullptr;
    double *yc64 = nullptr, *yi64 = nullptr, *yh64 = nullptr;
    float* yg32 = nullptr;  // FP32 copy of yc, gathered by the mixed-mode primal step
    double *prev_ax = nullptr, *prev_xh = nullptr;
    double *pi_x = nullptr, *pi_y = nullptr, *pi_xn = nullptr, *pi_part = nullptr;
    double *part_rows = nullptr, *part_cols = nullptr;
    // Anderson acceleration at restarts (anderson.cuh); aa_w = 0 when off.
    int aa_w = 0, aa_nb = 1;
    double *aa_X = nullptr, *aa_R = nullptr, *aa_out = nullptr, *aa_part = nullptr, *aa_gram = nullptr,
           *aa_work = nullptr;
    int* aa_order = nullptr;
    AaState* aa_st = nullptr;
    DevState* st = nullptr;
    DevConst* dc = nullptr;
    PowerState* ps = nullptr;
    DevState* h_st = nullptr;    // pinned mirror
    PowerState* h_ps = nullptr;  // pinned mirror

    cudaGraphExec_t cycle[2] = {nullptr, nullptr};
    int cycle_N[2] = {0, 0};
    cudaGraphExec_t power = nullptr;
    int launches_cycle[2] = {0, 0};
    int launches_power = 0;
    static constexpr int kPowerChunk = 8;

    ~DeviceLp() {
        for (auto& g : cycle)
            if (g) cudaGraphExecDestroy(g);
        for (auto& row : kev)
            for (auto& e : row)
                if (e) cudaEventDestroy(e);
        if (power) cudaGraphExecDestroy(power);
        if (arena) cudaFree(arena);
        if (h_st) cudaFreeHost(h_st);
        if (h_ps) cudaFreeHost(h_ps);
        if (stream) cudaStreamDestroy(stream);
    }

    IterArgs<float> iter32(const pdlpx_options& o) const {
        IterArgs<float> a{};
        a.at_ptr = at_ptr;
        a.at_idx = at_idx;
        a.at_val = at_v32;
        a.a_ptr = a_ptr;
        a.a_idx = a_idx;
        a.a_val = a_v32;
        a.cp = cp32;
        a.rp = rp32;
        a.xc = xc64;
        a.xi = xi32;
        a.xr = xr32;
        a.xh = xh32;
        a.yc = yc64;
        a.yg = yg32;
        a.yi = yi32;
        a.yh = yh32;
        a.st = st;
        a.m = m;
        a.n = n;
        a.max_iter = o.max_iter;
        a.polish_max_iter = o.polish_max_iter;
        a.N = o.termination_eval_frequency;
        return a;
    }
    IterArgs<double> iter64(const pdlpx_options& o) const {
        IterArgs<double> a{};
        a.at_ptr = at_ptr;
        a.at_idx = at_idx;
        a.at_val = at_v64;
        a.a_ptr = a_ptr;
        a.a_idx = a_idx;
        a.a_val = a_v64;
        a.cp = cp64;
        a.rp = rp64;
        a.xc = xc64;
        a.xi = xi64;
        a.xr = xr64;
        a.xh = xh64;
        a.yc = yc64;
        a.yg = yc64;
        a.yi = yi64;
        a.yh = yh64;
        a.st = st;
        a.m = m;
        a.n = n;
        a.max_iter = o.max_iter;
        a.polish_max_iter = o.polish_max_iter;
        a.N = o.termination_eval_frequency;
        return a;
    }
    AaArgs aaArgs(double reg) const {
        AaArgs a{};
        a.X = aa_X;
        a.Rr = aa_R;
        a.out = aa_out;
        a.part = aa_part;
        a.gram = aa_gram;
        a.work = aa_work;
        a.order = aa_order;
        a.as = aa_st;
        a.st = st;
        a.lb = lb64;
        a.ub = ub64;
        a.n = n;
        a.m = m;
        a.w = aa_w;
        a.nb = aa_nb;
        a.reg = reg;
        return a;
    }
    template <class T>
    CheckArgs<T> check(const T* xh, const T* xi, const T* yh, const T* yi) const {
        CheckArgs<T> c{};
        c.a_ptr = a_ptr;
        c.a_idx = a_idx;
        c.a_val = a_v64;
        c.at_ptr = at_ptr;
        c.at_idx = at_idx;
        c.at_val = at_v64;
        c.xh = xh;
        c.xi = xi;
        c.yh = yh;
        c.yi = yi;
        c.c64 = c64;
        c.lb64 = lb64;
        c.ub64 = ub64;
        c.cs64 = cs64;
        c.tau64 = tau64;
        c.rl64 = rl64;
        c.ru64 = ru64;
        c.rs64 = rs64;
        c.sig64 = sig64;
        c.prev_ax = prev_ax;
        c.prev_xh = prev_xh;
        c.part_rows = part_rows;
        c.part_cols = part_cols;
        c.dc = dc;
        c.st = st;
        c.m = m;
        c.n = n;
        return c;
    }
};

namespace {

template <class T>
IterArgs<T> iterArgs(const DeviceLp& d, const pdlpx_options& o);
template <>
IterArgs<float> iterArgs<float>(const DeviceLp& d, const pdlpx_options& o) {
    return d.iter32(o);
}
template <>
IterArgs<double> iterArgs<double>(const DeviceLp& d, const pdlpx_options& o) {
    return d.iter64(o);
}

// The FP32 copy of y that writers of yc keep (mixed mode), else null (in FP64
// mode the primal step gathers yc itself).
template <class T>
T* ygCopy(const IterArgs<T>& ia) {
    return sizeof(T) == 4 ? ia.yg : nullptr;
}

// Sliced-ELL values of a side in storage type T.
template <class T>
const T* sellVals(const DeviceLp& d, bool primal);
template <>
const float* sellVals<float>(const DeviceLp& d, bool primal) {
    return primal ? d.sp_v32 : d.sd_v32;
}
template <>
const double* sellVals<double>(const DeviceLp& d, bool primal) {
    return primal ? d.sp_v64 : d.sd_v64;
}

static int sellGrid(int64_t rows) { return static_cast<int>(std::max<int64_t>(1, (rows + kBlock - 1) / kBlock)); }

// A launch with programmatic stream serialization: the kernel may begin while
// the one before it on the stream finishes (it calls pdlWait before reading
// what that kernel writes).  Inside a stream capture the edge becomes a
// programmatic dependency of the graph.
template <class... KArgs, class... Args>
static cudaError_t launchPdl(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t s,
                            Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(static_cast<unsigned>(block));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Shared memory per block of a hot kernel running `minb` blocks per SM: the
// prefix's share of the SM, within the device limits (1 KB of each block's
// share is the runtime's).  Shared memory is carved out of the SM's L1, which
// also holds the sectors of the loads in flight, so the prefix's share is a
// trade between gathers served from shared memory and L1 room for the rest.
static int hotBlockBytes(const DeviceLp& d, int minb) {
    const int b = std::min({d.hot_smem_block, d.hot_smem_sm / minb - 1024, d.hot_bytes_sm / minb});
    return std::max(0, b & ~15);
}
template <class X>
static int hotCap(const DeviceLp& d, int minb) {
    return hotBlockBytes(d, minb) / static_cast<int>(sizeof(X));
}
// Hot prefix length of the primal (y) / dual (x_refl) gathers at precision T
// (both gathered as T); 0 when the side does not use a hot kernel.
template <class T>
static int hotPrimal(const DeviceLp& d) {
    return d.hotP > 0 ? std::min(d.hotP, hotCap<T>(d, sellMinBlocks<T, true>())) : 0;
}
template <class T>
static int hotDual(const DeviceLp& d) {
    return d.hotD > 0 ? std::min(d.hotD, hotCap<T>(d, sellMinBlocks<T>())) : 0;
}

// Dynamic shared memory limits of every hot kernel (set once per load).
template <class T>
static void setHotAttrs(const DeviceLp& d) {
    const int bp = hotBlockBytes(d, sellMinBlocks<T, true>()), bd = hotBlockBytes(d, sellMinBlocks<T>());
    for (int k = 0; k < kEngSell; ++k) {
        const int shape = kNumShapes + k;
        PDLPX_ENG_SELL_SWITCH(shape, {
            cudaFuncSetAttribute(primalSellHot<UU, T, SS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bp);
            cudaFuncSetAttribute(dualSellHot<UU, T, SS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bd);
        });
    }
}

// The step kernels use no shared memory; their scattered gathers lean on L1
// (the power-law LPs' popular columns hit there), so they ask for the largest
// L1 carve-out.
template <class T>
static void preferL1() {
    for (int k = 0; k < kEngSell; ++k) {
        const int shape = kNumShapes + k;
        PDLPX_ENG_SELL_SWITCH(shape, {
            cudaFuncSetAttribute(primalSellStep<UU, T, SS>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
            cudaFuncSetAttribute(dualSellStep<UU, T, SS>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
        });
    }
    for (int shape = 0; shape < kNumShapes; ++shape) {
        PDLPX_SHAPE_SWITCH(shape, {
            cudaFuncSetAttribute(primalStep<GG, RR, UU, T, true>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
            cudaFuncSetAttribute(dualStep<GG, RR, UU, T>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
        });
    }
}

// Short-row launch of one side in `shape` (CSR, or sliced ELL when isSell).
template <class T>
void launchPrimalShort(const DeviceLp& d, const IterArgs<T>& ia, int shape, int k, cudaStream_t s) {
    const int H = isSell(shape) ? hotPrimal<T>(d) : 0;
    if (H > 0) {
        const size_t bytes = static_cast<size_t>(H) * sizeof(T);
        PDLPX_ENG_SELL_SWITCH(shape, (primalSellHot<UU, T, SS>
                                      <<<sellGrid(d.n - d.nlP), kBlock, bytes, s>>>(
                                          ia, d.sp_hdr, d.sp_idx, sellVals<T>(d, true), k, d.nlP, d.n, H)));
    } else if (isSell(shape)) {
        PDLPX_ENG_SELL_SWITCH(shape, (primalSellStep<UU, T, SS><<<sellGrid(d.n - d.nlP), kBlock, 0, s>>>(
                                         ia, d.sp_hdr, d.sp_idx, sellVals<T>(d, true), k, d.nlP, d.n)));
    } else {
        PDLPX_SHAPE_SWITCH(shape, (primalStep<GG, RR, UU, T, true><<<gridForShape(d.n - d.nlP, shape), kBlock, 0, s>>>(
                                      ia, k, d.nlP, d.n)));
    }
}
template <class T>
void launchDualShort(const DeviceLp& d, const IterArgs<T>& ia, int shape, int k, cudaStream_t s) {
    const int H = isSell(shape) ? hotDual<T>(d) : 0;
    if (H > 0) {
        const size_t bytes = static_cast<size_t>(H) * sizeof(T);
        PDLPX_ENG_SELL_SWITCH(shape, (dualSellHot<UU, T, SS>
                                      <<<sellGrid(d.m - d.nlD), kBlock, bytes, s>>>(
                                          ia, d.sd_hdr, d.sd_idx, sellVals<T>(d, false), k, d.nlD, d.m, H)));
    } else if (isSell(shape)) {
        PDLPX_ENG_SELL_SWITCH(shape, (launchPdl(dualSellStep<UU, T, SS>, sellGrid(d.m - d.nlD), kBlock, 0, s, ia,
                                                d.sd_hdr, d.sd_idx, sellVals<T>(d, false), k, d.nlD, d.m)));
    } else {
        PDLPX_SHAPE_SWITCH(shape, (dualStep<GG, RR, UU, T><<<gridForShape(d.m - d.nlD, shape), kBlock, 0, s>>>(
                                      ia, k, d.nlD, d.m)));
    }
}

// Step launches of one iteration on each side: the long rows (if any), then the rest.
template <class T>
int launchPrimal(const DeviceLp& d, const IterArgs<T>& ia, int k, cudaStream_t s) {
    int n = 0;
    if constexpr (sizeof(T) == 4) {
        if (d.lt_C > 0) {
            const LongTileArgs t = d.tiles();
            launchPdl(primalLongTiles, d.lt_C * d.lt_G, kTileBlock, tileSmemBytes(d.lt_R, d.lt_maxcols), s, ia, t, k);
            ++n;
            if (d.n > d.nlP && isSell(d.shapeP) && hotPrimal<T>(d) == 0) {
                const int fb = sellGrid(d.nlP);
                PDLPX_ENG_SELL_SWITCH(d.shapeP, (launchPdl(primalSellFinish<UU, SS>, fb + sellGrid(d.n - d.nlP), kBlock, 0,
                                                           s, ia, d.sp_hdr, d.sp_idx, d.sp_v32, k, d.nlP, d.n, t, fb)));
                return n + 1;
            }
            primalLongFinish<<<sellGrid(d.nlP), kBlock, 0, s>>>(ia, t, k);
            ++n;
            if (d.n > d.nlP) {
                launchPrimalShort<T>(d, ia, d.shapeP, k, s);
                ++n;
            }
            return n;
        }
    }
    if (d.nlP > 0) {
        PDLPX_SHAPE_SWITCH(d.shapeLP,
                           (primalStep<GG, RR, UU, T, true><<<gridForShape(d.nlP, d.shapeLP), kBlock, 0, s>>>(ia, k, 0, d.nlP)));
        ++n;
    }
    if (d.n > d.nlP) {
        launchPrimalShort<T>(d, ia, d.shapeP, k, s);
        ++n;
    }
    return n;
}
template <class T>
int launchDual(const DeviceLp& d, const IterArgs<T>& ia, int k, cudaStream_t s) {
    int n = 0;
    if (d.nlD > 0) {
        PDLPX_SHAPE_SWITCH(d.shapeLD,
                           (dualStep<GG, RR, UU, T><<<gridForShape(d.nlD, d.shapeLD), kBlock, 0, s>>>(ia, k, 0, d.nlD)));
        ++n;
    }
    if (d.m > d.nlD) {
        launchDualShort<T>(d, ia, d.shapeD, k, s);
        ++n;
    }
    return n;
}
// FP64 check pass: short rows write partials [0, nb_*_s), long rows the rest.
template <class T>
int launchChecks(const DeviceLp& d, const CheckArgs<T>& ca, cudaStream_t s) {
    PDLPX_G_SWITCH(d.gA, (checkRows<GG, T><<<d.nb_rows_s, kBlock, 0, s>>>(ca, d.nlD, d.m, 0)));
    PDLPX_G_SWITCH(d.gAT, (checkCols<GG, T><<<d.nb_cols_s, kBlock, 0, s>>>(ca, d.nlP, d.n, 0)));
    int n = 2;
    if (d.nlD > 0) {
        PDLPX_G_SWITCH(d.gLA, (checkRows<GG, T><<<d.nb_rows - d.nb_rows_s, kBlock, 0, s>>>(ca, 0, d.nlD, d.nb_rows_s)));
        ++n;
    }
    if (d.nlP > 0) {
        PDLPX_G_SWITCH(d.gLAT, (checkCols<GG, T><<<d.nb_cols - d.nb_cols_s, kBlock, 0, s>>>(ca, 0, d.nlP, d.nb_cols_s)));
        ++n;
    }
    return n;
}

// One restart cycle: N fused iterations, check, controller, restart copy.
template <class T>
int launchCycle(DeviceLp& d, const pdlpx_options& o) {
    const IterArgs<T> ia = iterArgs<T>(d, o);
    const CheckArgs<T> ca = d.check<T>(ia.xh, ia.xi, ia.yh, ia.yi);
    cudaStream_t s = d.stream;
    int launches = 0;
    const int p = sizeof(T) == 8 ? 1 : 0;
    // Live step timing: under capture, an event recorded with the External flag
    // becomes an event-record node of the graph (a plain record would only
    // mark a dependency), so every replay records it on the device.
    auto mark = [&](cudaEvent_t e) { cudaEventRecordWithFlags(e, s, cudaEventRecordExternal); };
    for (int k = 1; k <= o.termination_eval_frequency; ++k) {
        const bool timed = k == d.kev_iter && d.kev[p][0] != nullptr;
        if (timed) mark(d.kev[p][0]);
        launches += launchPrimal<T>(d, ia, k, s);
        if (timed) mark(d.kev[p][1]);
        launches += launchDual<T>(d, ia, k, s);
        if (timed) mark(d.kev[p][2]);
    }
    launches += launchChecks<T>(d, ca, s) - 2;
    controller<<<1, kBlock, 0, s>>>(d.st, d.dc, d.part_rows, d.part_cols, sizeof(T) == 8 ? 1 : 0);
    const int nb = std::max(1, std::min(gridFor(std::max(d.m, d.n), 1), 8 * d.sms));
    const AaArgs aa = d.aaArgs(o.anderson_regularization);
    if (d.aa_w > 0) {
        aaStore<T><<<d.aa_nb, kBlock, 0, s>>>(aa, ia.xh, ia.xi, ia.yh, ia.yi);
        aaSolve<<<1, 32, 0, s>>>(aa);
        aaExtrapolate<<<d.aa_nb, kBlock, 0, s>>>(aa);
        aaDecide<<<1, 32, 0, s>>>(aa);
        launches += 4;
    }
    restartCopy<T><<<nb, kBlock, 0, s>>>(d.st, d.n, d.m, ia.xh, ia.yh, ia.xi, ia.yi, ia.xc, ia.yc,
                                         d.aa_w > 0 ? &d.aa_st->accepted : nullptr, ygCopy(ia));
    if (d.aa_w > 0) {
        aaApply<T><<<nb, kBlock, 0, s>>>(aa, ia.xi, ia.yi, ia.xc, ia.yc, ygCopy(ia));
        ++launches;
    }
    launches += 4;
    if (sizeof(T) == 4 && d.mixed) {
        PromoteArgs pa{d.xi32, d.xh32, d.yi32, d.yh32, d.xi64, d.xh64, d.yi64, d.yh64, d.st, d.n, d.m};
        promoteIterates<<<nb, kBlock, 0, s>>>(pa);
        finishPromote<<<1, 1, 0, s>>>(d.st);
        launches += 2;
    }
    return launches;
}

template <class V>
int launchPowerChunk(DeviceLp& d, const PowerArgs& pa, const PowerMat<V>& mt, int chunk) {
    cudaStream_t s = d.stream;
    int launches = 0;
    for (int it = 0; it < chunk; ++it) {
        // A x for every row before A^T y reads it
        if (isSell(d.shapeD))
            powerASell<V><<<sellGrid(d.m - d.nlD), kBlock, 0, s>>>(pa, d.sd_hdr, d.sd_idx, sellVals<V>(d, false),
                                                                   d.nlD, d.m);
        else
            PDLPX_G_SWITCH(d.gA, (powerA<GG, V><<<gridFor(d.m - d.nlD, d.gA), kBlock, 0, s>>>(pa, mt, d.nlD, d.m)));
        if (d.nlD > 0) {
            PDLPX_G_SWITCH(d.gLA, (powerA<GG, V><<<gridFor(d.nlD, d.gLA), kBlock, 0, s>>>(pa, mt, 0, d.nlD)));
            ++launches;
        }
        if (isSell(d.shapeP))
            powerAtSell<V><<<d.nb_pi_s, kBlock, 0, s>>>(pa, d.sp_hdr, d.sp_idx, sellVals<V>(d, true), d.nlP, d.n, 0);
        else
            PDLPX_G_SWITCH(d.gAT, (powerAt<GG, V><<<d.nb_pi_s, kBlock, 0, s>>>(pa, mt, d.nlP, d.n, 0)));
        if (d.nlP > 0) {
            PDLPX_G_SWITCH(d.gLAT, (powerAt<GG, V><<<d.nb_pi - d.nb_pi_s, kBlock, 0, s>>>(pa, mt, 0, d.nlP, d.nb_pi_s)));
            ++launches;
        }
        powerFinish1<<<1, kBlock, 0, s>>>(pa);
        powerNormalize<<<d.nb_pi, kBlock, 0, s>>>(pa);
        powerFinish2<<<1, kBlock, 0, s>>>(pa);
        launches += 5;
    }
    return launches;
}

template <class T>
void packCols(const ScaledLp& sc, std::vector<ColPack<T>>& out) {
    out.resize(sc.c.size());
    for (size_t j = 0; j < sc.c.size(); ++j)
        out[j] = ColPack<T>{static_cast<T>(sc.c[j]), static_cast<T>(sc.cl[j]), static_cast<T>(sc.cu[j]),
                            static_cast<T>(sc.tau[j])};
}
template <class T>
void packRows(const ScaledLp& sc, std::vector<RowPack<T>>& out) {
    out.resize(sc.rl.size());
    for (size_t i = 0; i < sc.rl.size(); ++i)
        out[i] = RowPack<T>{static_cast<T>(sc.sigma[i]), static_cast<T>(sc.rl[i]), static_cast<T>(sc.ru[i]),
                            static_cast<T>(sc.row_type[i])};
}

// Vectors between the original numbering and the device numbering
// (pos: original -> device; empty = identity).
void toDevice(std::vector<double>& v, const std::vector<int32_t>& pos) {
    if (pos.empty()) return;
    std::vector<double> w(v.size());
    for (size_t k = 0; k < v.size(); ++k) w[pos[k]] = v[k];
    v.swap(w);
}
void fromDevice(std::vector<double>& v, const std::vector<int32_t>& pos) {
    if (pos.empty()) return;
    std::vector<double> w(v.size());
    for (size_t k = 0; k < v.size(); ++k) w[k] = v[pos[k]];
    v.swap(w);
}

bool timeUp(std::chrono::steady_clock::time_point t0, double lim) {
    if (lim < 0.0) return false;
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >= lim;
}

}  // namespace

// f(begin, end) over contiguous blocks of [0, count) on up to 16 host threads
// (one below 1M entries of `work`); the blocks write disjoint output.
template <class F>
static void hostBlocks(size_t work, int64_t count, F&& f) {
    const int nt = work < (size_t(1) << 20)
                       ? 1
                       : static_cast<int>(std::min<int64_t>(
                             count, std::max(1u, std::min(16u, std::thread::hardware_concurrency()))));
    if (nt <= 1) {
        f(int64_t{0}, count);
        return;
    }
    std::vector<std::thread> ts;
    for (int t = 0; t < nt; ++t) ts.emplace_back([&, t] { f(count * t / nt, count * (t + 1) / nt); });
    for (auto& th : ts) th.join();
}

// out = the FP32 roundings of v, on host threads for large arrays.
static void toFloat(const std::vector<double>& v, std::vector<float>& out) {
    out.resize(v.size());
    const int64_t n = static_cast<int64_t>(v.size());
    hostBlocks(v.size(), n, [&](int64_t b, int64_t e) {
        for (int64_t k = b; k < e; ++k) out[static_cast<size_t>(k)] = static_cast<float>(v[static_cast<size_t>(k)]);
    });
}

// Device numbering of one matrix side's rows.  Rows far longer than the rest
// (more entries than max(64, 8 x the mean)) come first, longest first; the
// other rows follow -- sorted by length (longest first, stable) inside windows
// of `window` rows (option sell_window; by default the whole side) when the
// side is stored as sliced ELL, else in their original order.  Sorting puts
// rows of nearly equal length into each 32-row slice (on the 500k x 2M
// power-law LP 5 % padding), hands the block scheduler the heaviest slices
// first, and, over the whole side, puts the most-gathered rows of a power-law
// LP next to each other in the vector the other side gathers.  Measured on that
// LP (B200, live step times, primal / dual): windows of 4,096 rows 115.0 /
// 78.7 us, whole-side order for the columns 94.4 / 75.0, for the rows 116.2 /
// 71.8, for both 96.5 / 68.4 (solve 12.61 -> 10.54 s).  A window keeps every
// row within `window` places of where it was, for LPs whose original numbering
// gives the other side's gathers locality.  `sell_opt` is the option (-1 automatic: sliced ELL when the
// short rows' mean length is at most 64; 1 whenever there are short rows;
// 0 never); `sell` receives the decision.  Returns the number of long rows;
// `order` stays empty for the identity.
static int32_t sideOrder(const Csr& a, int sell_opt, bool& sell, std::vector<int32_t>& order, int64_t window) {
    order.clear();
    sell = false;
    const int32_t rows = a.rows;
    if (rows == 0) return 0;
    const double mean = static_cast<double>(a.nnz()) / rows;
    const int32_t thr = std::max<int32_t>(64, static_cast<int32_t>(8.0 * mean));
    std::vector<int32_t> lng, sht;
    int64_t zs = 0;
    for (int32_t i = 0; i < rows; ++i) {
        const int32_t len = a.ptr[i + 1] - a.ptr[i];
        if (len > thr) {
            lng.push_back(i);
        } else {
            sht.push_back(i);
            zs += len;
        }
    }
    auto len = [&](int32_t x) { return a.ptr[x + 1] - a.ptr[x]; };
    if (!sht.empty())
        sell = sell_opt > 0 || (sell_opt < 0 && static_cast<double>(zs) <= 64.0 * static_cast<double>(sht.size()));
    if (sell && static_cast<int64_t>(sht.size()) <= window) {
        // one window: a stable counting sort by length (short rows have at
        // most thr entries), the same order as the stable comparison sort
        std::vector<int64_t> start(static_cast<size_t>(thr) + 2, 0);
        for (int32_t x : sht) ++start[static_cast<size_t>(thr - len(x)) + 1];
        for (size_t q = 1; q < start.size(); ++q) start[q] += start[q - 1];
        std::vector<int32_t> out(sht.size());
        for (int32_t x : sht) out[static_cast<size_t>(start[static_cast<size_t>(thr - len(x))]++)] = x;
        sht.swap(out);
    } else if (sell) {
        const int64_t windows = (static_cast<int64_t>(sht.size()) + window - 1) / window;
        hostBlocks(sht.size() * 16, windows, [&](int64_t w0, int64_t w1) {
            for (int64_t w = w0; w < w1; ++w) {
                const size_t b = static_cast<size_t>(w) * window, e = std::min(sht.size(), b + static_cast<size_t>(window));
                std::stable_sort(sht.begin() + b, sht.begin() + e, [&](int32_t x, int32_t y) { return len(x) > len(y); });
            }
        });
    }
    std::stable_sort(lng.begin(), lng.end(), [&](int32_t x, int32_t y) { return len(x) > len(y); });
    bool identity = true;
    for (size_t k = 0; k < sht.size() && identity; ++k) identity = sht[k] == static_cast<int32_t>(lng.size() + k);
    if (lng.empty() && identity) return 0;
    order = lng;
    order.insert(order.end(), sht.begin(), sht.end());
    return static_cast<int32_t>(lng.size());
}

// Sliced ELL of rows [r0, a.rows) of a (device numbering): slice s holds rows
// r0 + 32 s .. r0 + 32 s + 31, entry k of lane l at hdr[s].x + 32 k + l, padded
// with index 0 / value 0 to the slice's longest row (hdr[s].y).  False when the
// padded entries would not fit 32-bit offsets (the side then keeps CSR).
struct SellHost {
    std::vector<int2> hdr;
    std::vector<int32_t> idx;
    std::vector<double> val;
};
static bool buildSell(const Csr& a, int32_t r0, SellHost& h) {
    const int64_t rows = static_cast<int64_t>(a.rows) - r0;
    const int64_t slices = (rows + kSlice - 1) / kSlice;
    h.hdr.resize(static_cast<size_t>(slices));
    int64_t e = 0;
    for (int64_t s = 0; s < slices; ++s) {
        int32_t w = 0;
        for (int64_t r = s * kSlice; r < std::min<int64_t>(rows, (s + 1) * kSlice); ++r)
            w = std::max(w, a.ptr[r0 + r + 1] - a.ptr[r0 + r]);
        h.hdr[static_cast<size_t>(s)] = make_int2(static_cast<int>(e), w);
        e += static_cast<int64_t>(w) * kSlice;
        if (e > std::numeric_limits<int32_t>::max()) return false;
    }
    h.idx.assign(static_cast<size_t>(e), 0);
    h.val.assign(static_cast<size_t>(e), 0.0);
    // slices own disjoint entry ranges: fill them in parallel blocks of slices
    hostBlocks(static_cast<size_t>(e), slices, [&](int64_t s0, int64_t s1) {
        for (int64_t r = s0 * kSlice; r < std::min<int64_t>(rows, s1 * kSlice); ++r) {
            const int64_t first = h.hdr[static_cast<size_t>(r / kSlice)].x + (r % kSlice);
            const int32_t b = a.ptr[r0 + r], cnt = a.ptr[r0 + r + 1] - b;
            for (int32_t k = 0; k < cnt; ++k) {
                const size_t at = static_cast<size_t>(first + static_cast<int64_t>(k) * kSlice);
                h.idx[at] = a.idx[b + k];
                h.val[at] = a.val[b + k];
            }
        }
    });
    return true;
}

// Long columns [0, nl) of A^T (device numbering) in row chunks for the tiled
// primal step (primalLongTiles): chunk c holds rows [c R, (c + 1) R), R a
// multiple of 16 (so each chunk of y starts on a 16-byte boundary) and at most
// max_rows; entries of column j in chunk c keep their CSR order; G column
// groups per chunk (as many tiles as SMs, so the tiles run in one wave of one
// block per SM; at least one group), cut at equal weights (entries + 8 per
// column).  False when a chunk offset would not fit 16 bits or a tile's shared
// memory would exceed smem_max.
struct LongTilesHost {
    int R = 0, C = 0, G = 0, maxcols = 0;
    std::vector<int32_t> off, gb;
    std::vector<uint16_t> row;
    std::vector<float> val;
};
static bool buildLongTiles(const Csr& at, int32_t nl, int32_t m, int sms, int max_rows, size_t smem_max,
                           LongTilesHost& t) {
    if (nl <= 0 || m <= 0) return false;
    int C = (m + max_rows - 1) / max_rows;
    const int R = (((m + C - 1) / C) + 15) & ~15;
    C = (m + R - 1) / R;
    if (R > 65536) return false;
    t.R = R;
    t.C = C;
    t.G = std::max(1, std::min(nl, sms / C));
    const size_t cells = static_cast<size_t>(C) * static_cast<size_t>(nl);
    t.off.assign(cells + 1, 0);
    for (int32_t j = 0; j < nl; ++j)
        for (int32_t k = at.ptr[j]; k < at.ptr[j + 1]; ++k)
            ++t.off[static_cast<size_t>(at.idx[k] / R) * nl + j + 1];
    for (size_t q = 0; q < cells; ++q) t.off[q + 1] += t.off[q];
    const int64_t z = at.ptr[nl];
    t.row.resize(static_cast<size_t>(z));
    t.val.resize(static_cast<size_t>(z));
    std::vector<int32_t> pos(t.off.begin(), t.off.end() - 1);
    for (int32_t j = 0; j < nl; ++j)
        for (int32_t k = at.ptr[j]; k < at.ptr[j + 1]; ++k) {
            const int32_t c = at.idx[k] / R;
            const int32_t p = pos[static_cast<size_t>(c) * nl + j]++;
            t.row[p] = static_cast<uint16_t>(at.idx[k] - c * R);
            t.val[p] = static_cast<float>(at.val[k]);
        }
    // groups of equal weight (entries + 8 per column, the per-column work of a
    // lane group in entries)
    const int64_t wtot = z + 8 * static_cast<int64_t>(nl);
    t.gb.assign(1, 0);
    int64_t w = 0;
    for (int32_t j = 0; j < nl; ++j) {
        w += (at.ptr[j + 1] - at.ptr[j]) + 8;
        const int64_t target = wtot * static_cast<int64_t>(t.gb.size()) / t.G;
        if (j + 1 < nl && static_cast<int>(t.gb.size()) < t.G && w >= target) t.gb.push_back(j + 1);
    }
    t.gb.push_back(nl);
    t.G = static_cast<int>(t.gb.size()) - 1;
    t.maxcols = 0;
    for (int g = 0; g < t.G; ++g) t.maxcols = std::max(t.maxcols, t.gb[g + 1] - t.gb[g]);
    return tileSmemBytes(t.R, t.maxcols) <= smem_max;
}

// Sliced-ELL shape of a side from the options: a pinned sliced-ELL shape
// (kNumShapes + 1 .. kNumShapes + kNumSell), else 4 entries per round for mean
// lengths up to 12 and 8 above (the packed batch's measured picks).
static int sellShape(int pinned, int64_t nnz, int32_t rows) {
    if (pinned > kNumShapes && pinned <= kNumShapes + kEngSell) return pinned - 1;
    const double mean = rows > 0 ? static_cast<double>(nnz) / rows : 0.0;
    return kNumShapes + (mean <= 12.0 ? 0 : 1);
}

// The scaled LP with its rows in order `ro` and columns in order `co` (new
// position -> original; empty = identity); rpos / cpos receive original ->
// new.  Entries keep their place inside their row.
static void permuteScaled(const ScaledLp& sc, const std::vector<int32_t>& ro, const std::vector<int32_t>& co,
                          ScaledLp& out, std::vector<int32_t>& rpos, std::vector<int32_t>& cpos) {
    const int32_t m = sc.a.rows, n = sc.a.cols;
    auto inverse = [](const std::vector<int32_t>& ord, int32_t k, std::vector<int32_t>& pos) {
        pos.resize(k);
        for (int32_t q = 0; q < k; ++q) pos[ord.empty() ? q : ord[q]] = q;
    };
    inverse(ro, m, rpos);
    inverse(co, n, cpos);
    auto oldRow = [&](int32_t i) { return ro.empty() ? i : ro[i]; };
    auto oldCol = [&](int32_t j) { return co.empty() ? j : co[j]; };
    out.obj_sign = sc.obj_sign;
    out.obj_scale = sc.obj_scale;
    out.con_scale = sc.con_scale;
    out.precond_pw = sc.precond_pw;
    // new row r is old row ord[r] with its indices renumbered; rows are copied
    // in parallel blocks once the pointers are known
    auto permuteCsr = [](const Csr& a, int32_t rows, int32_t cols, const std::vector<int32_t>& ord,
                         const std::vector<int32_t>& idxPos, Csr& b) {
        auto old = [&](int32_t r) { return ord.empty() ? r : ord[r]; };
        b.rows = rows;
        b.cols = cols;
        b.ptr.resize(static_cast<size_t>(rows) + 1);
        b.ptr[0] = 0;
        for (int32_t r = 0; r < rows; ++r) b.ptr[r + 1] = b.ptr[r] + (a.ptr[old(r) + 1] - a.ptr[old(r)]);
        b.idx.resize(a.idx.size());
        b.val.resize(a.val.size());
        hostBlocks(a.idx.size(), rows, [&](int64_t r0, int64_t r1) {
            for (int64_t r = r0; r < r1; ++r) {
                const int32_t o = old(static_cast<int32_t>(r));
                int32_t p = b.ptr[r];
                for (int32_t k = a.ptr[o]; k < a.ptr[o + 1]; ++k, ++p) {
                    b.idx[p] = idxPos[a.idx[k]];
                    b.val[p] = a.val[k];
                }
            }
        });
    };
    permuteCsr(sc.a, m, n, ro, cpos, out.a);
    permuteCsr(sc.at, n, m, co, rpos, out.at);
    auto cols = [&](const std::vector<double>& v, std::vector<double>& w) {
        w.resize(n);
        for (int32_t j = 0; j < n; ++j) w[j] = v[oldCol(j)];
    };
    auto rowsOf = [&](const std::vector<double>& v, std::vector<double>& w) {
        w.resize(m);
        for (int32_t i = 0; i < m; ++i) w[i] = v[oldRow(i)];
    };
    cols(sc.c, out.c);
    cols(sc.cl, out.cl);
    cols(sc.cu, out.cu);
    cols(sc.col_scale, out.col_scale);
    cols(sc.tau, out.tau);
    rowsOf(sc.rl, out.rl);
    rowsOf(sc.ru, out.ru);
    rowsOf(sc.row_scale, out.row_scale);
    rowsOf(sc.sigma, out.sigma);
    out.row_type.resize(m);
    for (int32_t i = 0; i < m; ++i) out.row_type[i] = sc.row_type[oldRow(i)];
}

// Launch shape of the long rows of one side, from their mean length.
static int longShape(int64_t nnz, int32_t rows) {
    const double mean = rows > 0 ? static_cast<double>(nnz) / rows : 0.0;
    if (mean <= 128) return 9;   // G=32
    if (mean <= 384) return 11;  // G=64
    if (mean <= 768) return 13;  // G=128, U=8
    return 15;                   // G=256, U=8
}

// Mixed mode stores the matrix and anchors in FP32 to halve the HBM bytes of
// the step kernels.  An LP whose FP64 working set per iteration is under
// 16 MB stays in L2 and saves no time by it -- the 2,000 x 5,000 random LP's
// FP64 step kernels measured as fast as its FP32 ones on B200 (8.1 vs 8.2 us
// primal, 8.3 vs 10.2 us dual) -- while the FP32 values cost accuracy, so such
// an LP runs the FP64 kernels from the start, unless fp64_switch = 0 asks for
// the FP32 kernels throughout.
constexpr int64_t kMixedMinBytes = int64_t(16) << 20;
static bool wantMixed(const pdlpx_options& o, int64_t m, int64_t n, int64_t nnz) {
    if (o.precision == PDLPX_PREC_FP64) return false;
    if (!o.fp64_switch) return true;
    return 24 * nnz + 64 * n + 56 * m >= kMixedMinBytes;
}

// Build (or rebuild) the device image of the scaled LP.
static int32_t buildDevice(std::unique_ptr<DeviceLp>& dp, const ScaledLp& sc_in, const pdlpx_options& o,
                           std::string& err) {
    const auto tb0 = std::chrono::steady_clock::now();
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        err = "no CUDA device visible";
        return PDLPX_E_NO_DEVICE;
    }
    const int dev = (o.device >= 0 && o.device < count) ? o.device : 0;
    PDLPX_CK(cudaSetDevice(dev));
    dp.reset(new DeviceLp());
    DeviceLp& d = *dp;
    d.device = dev;
    PDLPX_CK(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
    PDLPX_CK(cudaDeviceGetAttribute(&d.hot_smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    PDLPX_CK(cudaDeviceGetAttribute(&d.hot_smem_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    PDLPX_CK(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking));
    // Device numbering: long rows first, sliced-ELL sides' short rows sorted by
    // length (identity where neither applies).  A side whose shape or lane
    // count is pinned to CSR keeps CSR.
    std::vector<int32_t> ro, co;
    const int sellD_opt = (o.spmv_group_a > 0 || (o.shape_dual > 0 && o.shape_dual <= kNumShapes)) ? 0
                          : o.shape_dual > kNumShapes                                         ? 1
                                                                                               : o.sell;
    const int sellP_opt = (o.spmv_group_at > 0 || (o.shape_primal > 0 && o.shape_primal <= kNumShapes)) ? 0
                          : o.shape_primal > kNumShapes                                           ? 1
                                                                                                   : o.sell;
    bool sellD = false, sellP = false;
    const int64_t window = o.sell_window > 0 ? o.sell_window : std::numeric_limits<int32_t>::max();
    d.nlD = sideOrder(sc_in.a, sellD_opt, sellD, ro, window);
    d.nlP = sideOrder(sc_in.at, sellP_opt, sellP, co, window);
    const bool perm = !ro.empty() || !co.empty();
    ScaledLp permuted;
    if (perm) permuteScaled(sc_in, ro, co, permuted, d.rpos, d.cpos);
    const ScaledLp& sc = perm ? permuted : sc_in;
    if (ro.empty()) d.rpos.clear();
    if (co.empty()) d.cpos.clear();
    const auto tbp = std::chrono::steady_clock::now();
    SellHost hsP, hsD;
    if (sellP && !buildSell(sc.at, d.nlP, hsP)) sellP = false;
    if (sellD && !buildSell(sc.a, d.nlD, hsD)) sellD = false;
    const auto tbs = std::chrono::steady_clock::now();
    d.m = sc.a.rows;
    d.n = sc.a.cols;
    d.nnz = sc.a.nnz();
    d.mixed = wantMixed(o, sc.a.rows, sc.a.cols, sc.a.nnz());
    const int64_t m = d.m, n = d.n, nnz = d.nnz;
    const int64_t zlD = d.nlD > 0 ? sc.a.ptr[d.nlD] : 0, zlP = d.nlP > 0 ? sc.at.ptr[d.nlP] : 0;
    d.zlD = zlD;
    d.zlP = zlP;
    LongTilesHost ltH;
    // automatic: when the long columns hold at least 1.5 times as many entries
    // per SM as a chunk has rows (each tile's copy of y then serves >= 1.5
    // gathers per row it copies).  Measured on B200: the 500k x 2M power-law
    // LP's primal step 125.0 -> 117.5 us (58k entries per tile, 27.8k rows per
    // chunk: 2.1); the 100k x 400k one 45.9 -> 66.0 us (11k entries per tile,
    // 25k rows: 0.44).
    const int64_t chunks = d.m > 0 ? (d.m + kTileMaxRows - 1) / kTileMaxRows : 1;
    const int64_t chunk_rows = (((d.m + chunks - 1) / chunks) + 15) & ~int64_t(15);
    const bool want_tiles =
        o.long_tiles > 0 || (o.long_tiles < 0 && 2 * zlP >= 3 * static_cast<int64_t>(d.sms) * chunk_rows);
    if (d.mixed && want_tiles &&
        buildLongTiles(sc.at, d.nlP, d.m, d.sms, kTileMaxRows, static_cast<size_t>(d.hot_smem_block), ltH)) {
        d.lt_R = ltH.R;
        d.lt_C = ltH.C;
        d.lt_G = ltH.G;
        d.lt_maxcols = ltH.maxcols;
    }
    const auto tbt = std::chrono::steady_clock::now();
    const int32_t msD = d.m - d.nlD, msP = d.n - d.nlP;  // short rows
    d.gA = o.spmv_group_a > 0 ? o.spmv_group_a : pickGroup(nnz - zlD, msD);
    d.gAT = o.spmv_group_at > 0 ? o.spmv_group_at : pickGroup(nnz - zlP, msP);
    d.shapeD = sellD ? sellShape(o.shape_dual, nnz - zlD, msD) : chooseShape(o.shape_dual, o.spmv_group_a, nnz - zlD, msD);
    d.shapeP = sellP ? sellShape(o.shape_primal, nnz - zlP, msP)
                     : chooseShape(o.shape_primal, o.spmv_group_at, nnz - zlP, msP);
    d.gLA = d.nlD > 0 ? std::min(256, pickGroup(zlD, d.nlD)) : 1;
    d.gLAT = d.nlP > 0 ? std::min(256, pickGroup(zlP, d.nlP)) : 1;
    d.shapeLD = longShape(zlD, d.nlD);
    d.shapeLP = longShape(zlP, d.nlP);
    // Hot prefixes (option): the dual step gathers x, whose long columns
    // [0, nlP) come first; the primal step gathers y, long rows [0, nlD).
    const bool hot = o.hot_cache > 0;
    d.hot_bytes_sm = hot ? 1024 * o.hot_cache : 0;
    d.hotD = (hot && sellD && d.nlP > 0) ? d.nlP : 0;
    d.hotP = (hot && sellP && d.nlD > 0) ? d.nlD : 0;
    if (d.hotD > 0 || d.hotP > 0) {
        setHotAttrs<float>(d);
        setHotAttrs<double>(d);
    }
    preferL1<float>();
    preferL1<double>();
    const int cap = 4 * d.sms;
    d.nb_rows_s = std::max(1, std::min(gridFor(msD, d.gA), cap));
    d.nb_cols_s = std::max(1, std::min(gridFor(msP, d.gAT), cap));
    d.nb_rows = d.nb_rows_s + (d.nlD > 0 ? std::max(1, std::min(gridFor(d.nlD, d.gLA), cap)) : 0);
    d.nb_cols = d.nb_cols_s + (d.nlP > 0 ? std::max(1, std::min(gridFor(d.nlP, d.gLAT), cap)) : 0);
    d.nb_pi_s = d.nb_cols_s;
    d.nb_pi = d.nb_cols;

    // Arena layout.
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off += (bytes + 255) & ~static_cast<size_t>(255);
        return at;
    };
    const bool mixed = d.mixed;
    const size_t o_a_ptr = take(4 * (m + 1)), o_a_idx = take(4 * nnz), o_at_ptr = take(4 * (n + 1)),
                 o_at_idx = take(4 * nnz);
    const size_t o_a_v64 = take(8 * nnz), o_at_v64 = take(8 * nnz);
    const size_t o_a_v32 = mixed ? take(4 * nnz) : 0, o_at_v32 = mixed ? take(4 * nnz) : 0;
    const size_t o_cp32 = mixed ? take(16 * n) : 0, o_rp32 = mixed ? take(16 * m) : 0;
    const size_t o_cp64 = take(32 * n), o_rp64 = take(32 * m);
    const size_t o_c64 = take(8 * n), o_lb64 = take(8 * n), o_ub64 = take(8 * n), o_cs64 = take(8 * n),
                 o_tau64 = take(8 * n);
    const size_t o_rl64 = take(8 * m), o_ru64 = take(8 * m), o_rs64 = take(8 * m), o_sig64 = take(8 * m);
    size_t o_x32[3] = {0, 0, 0}, o_y32[3] = {0, 0, 0};
    if (mixed) {
        for (auto& v : o_x32) v = take(4 * n);
        for (auto& v : o_y32) v = take(4 * m);
    }
    size_t o_x64[4], o_y64[3];
    for (auto& v : o_x64) v = take(8 * n);
    for (auto& v : o_y64) v = take(8 * m);
    const bool adaptive = o.adaptive_step != 0;
    const size_t o_prev_ax = adaptive ? take(8 * m) : 0, o_prev_xh = adaptive ? take(8 * n) : 0;
    const size_t o_pi_x = take(8 * n), o_pi_y = take(8 * m), o_pi_xn = take(8 * n),
                 o_pi_part = take(8 * 2 * d.nb_pi);
    const size_t o_prow = take(8 * kRowSlots * d.nb_rows), o_pcol = take(8 * kColSlots * d.nb_cols);
    // sliced-ELL sides: slice headers, indices, FP64 values, FP32 values (mixed)
    const size_t eP = hsP.idx.size(), eD = hsD.idx.size();
    const size_t o_sp_hdr = sellP ? take(8 * hsP.hdr.size()) : 0, o_sp_idx = sellP ? take(4 * eP) : 0,
                 o_sp_v64 = sellP ? take(8 * eP) : 0, o_sp_v32 = sellP && mixed ? take(4 * eP) : 0;
    const size_t o_sd_hdr = sellD ? take(8 * hsD.hdr.size()) : 0, o_sd_idx = sellD ? take(4 * eD) : 0,
                 o_sd_v64 = sellD ? take(8 * eD) : 0, o_sd_v32 = sellD && mixed ? take(4 * eD) : 0;
    // long columns in row chunks: offsets, group bounds, rows, FP32 values, partials
    const bool lt = d.lt_C > 0;
    const size_t zt = ltH.row.size();
    const size_t o_lt_off = lt ? take(4 * ltH.off.size()) : 0, o_lt_gb = lt ? take(4 * ltH.gb.size()) : 0,
                 o_lt_row = lt ? take(2 * zt) : 0, o_lt_val = lt ? take(4 * zt) : 0,
                 o_lt_part = lt ? take(8 * static_cast<size_t>(d.nlP) * static_cast<size_t>(d.lt_C)) : 0;
    // Anderson ring (2 w (n + m) doubles), extrapolation scratch, partials, Gram matrix.
    d.aa_w = o.anderson_acceleration && o.anderson_window_size >= 2 ? o.anderson_window_size : 0;
    const size_t dim = static_cast<size_t>(n) + static_cast<size_t>(m);
    size_t o_aa[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (d.aa_w > 0) {
        const size_t w = static_cast<size_t>(d.aa_w);
        d.aa_nb = std::max(1, std::min(gridFor(static_cast<int64_t>(dim), 1), 4 * d.sms));
        o_aa[0] = take(8 * w * dim);
        o_aa[1] = take(8 * w * dim);
        o_aa[2] = take(8 * dim);
        o_aa[3] = take(8 * static_cast<size_t>(d.aa_nb) * std::max<size_t>(w, 2));
        o_aa[4] = take(8 * w * w);
        o_aa[5] = take(8 * (2 * w * w + 2 * w));
        o_aa[6] = take(4 * w);
        o_aa[7] = take(sizeof(AaState));
    }
    const size_t o_st = take(sizeof(DevState)), o_dc = take(sizeof(DevConst)), o_ps = take(sizeof(PowerState));
    d.arena_bytes = off;
    const auto tb1 = std::chrono::steady_clock::now();
    PDLPX_CK(cudaMalloc(reinterpret_cast<void**>(&d.arena), d.arena_bytes));
    PDLPX_CK(cudaMallocHost(reinterpret_cast<void**>(&d.h_st), sizeof(DevState)));
    PDLPX_CK(cudaMallocHost(reinterpret_cast<void**>(&d.h_ps), sizeof(PowerState)));
    char* b = d.arena;
    d.a_ptr = reinterpret_cast<int*>(b + o_a_ptr);
    d.a_idx = reinterpret_cast<int*>(b + o_a_idx);
    d.at_ptr = reinterpret_cast<int*>(b + o_at_ptr);
    d.at_idx = reinterpret_cast<int*>(b + o_at_idx);
    d.a_v64 = reinterpret_cast<double*>(b + o_a_v64);
    d.at_v64 = reinterpret_cast<double*>(b + o_at_v64);
    if (mixed) {
        d.a_v32 = reinterpret_cast<float*>(b + o_a_v32);
        d.at_v32 = reinterpret_cast<float*>(b + o_at_v32);
        d.cp32 = reinterpret_cast<ColPack<float>*>(b + o_cp32);
        d.rp32 = reinterpret_cast<RowPack<float>*>(b + o_rp32);
        d.xi32 = reinterpret_cast<float*>(b + o_x32[0]);
        d.xr32 = reinterpret_cast<float*>(b + o_x32[1]);
        d.xh32 = reinterpret_cast<float*>(b + o_x32[2]);
        d.yi32 = reinterpret_cast<float*>(b + o_y32[0]);
        d.yh32 = reinterpret_cast<float*>(b + o_y32[1]);
        d.yg32 = reinterpret_cast<float*>(b + o_y32[2]);
    }
    d.cp64 = reinterpret_cast<ColPack<double>*>(b + o_cp64);
    d.rp64 = reinterpret_cast<RowPack<double>*>(b + o_rp64);
    d.c64 = reinterpret_cast<double*>(b + o_c64);
    d.lb64 = reinterpret_cast<double*>(b + o_lb64);
    d.ub64 = reinterpret_cast<double*>(b + o_ub64);
    d.cs64 = reinterpret_cast<double*>(b + o_cs64);
    d.tau64 = reinterpret_cast<double*>(b + o_tau64);
    d.rl64 = reinterpret_cast<double*>(b + o_rl64);
    d.ru64 = reinterpret_cast<double*>(b + o_ru64);
    d.rs64 = reinterpret_cast<double*>(b + o_rs64);
    d.sig64 = reinterpret_cast<double*>(b + o_sig64);
    d.xc64 = reinterpret_cast<double*>(b + o_x64[0]);
    d.xi64 = reinterpret_cast<double*>(b + o_x64[1]);
    d.xr64 = reinterpret_cast<double*>(b + o_x64[2]);
    d.xh64 = reinterpret_cast<double*>(b + o_x64[3]);
    d.yc64 = reinterpret_cast<double*>(b + o_y64[0]);
    d.yi64 = reinterpret_cast<double*>(b + o_y64[1]);
    d.yh64 = reinterpret_cast<double*>(b + o_y64[2]);
    if (adaptive) {
        d.prev_ax = reinterpret_cast<double*>(b + o_prev_ax);
        d.prev_xh = reinterpret_cast<double*>(b + o_prev_xh);
    }
    d.pi_x = reinterpret_cast<double*>(b + o_pi_x);
    d.pi_y = reinterpret_cast<double*>(b + o_pi_y);
    d.pi_xn = reinterpret_cast<double*>(b + o_pi_xn);
    d.pi_part = reinterpret_cast<double*>(b + o_pi_part);
    d.part_rows = reinterpret_cast<double*>(b + o_prow);
    d.part_cols = reinterpret_cast<double*>(b + o_pcol);
    if (sellP) {
        d.sp_hdr = reinterpret_cast<int2*>(b + o_sp_hdr);
        d.sp_idx = reinterpret_cast<int*>(b + o_sp_idx);
        d.sp_v64 = reinterpret_cast<double*>(b + o_sp_v64);
        if (mixed) d.sp_v32 = reinterpret_cast<float*>(b + o_sp_v32);
    }
    if (sellD) {
        d.sd_hdr = reinterpret_cast<int2*>(b + o_sd_hdr);
        d.sd_idx = reinterpret_cast<int*>(b + o_sd_idx);
        d.sd_v64 = reinterpret_cast<double*>(b + o_sd_v64);
        if (mixed) d.sd_v32 = reinterpret_cast<float*>(b + o_sd_v32);
    }
    if (lt) {
        d.lt_off = reinterpret_cast<int32_t*>(b + o_lt_off);
        d.lt_gb = reinterpret_cast<int32_t*>(b + o_lt_gb);
        d.lt_row = reinterpret_cast<uint16_t*>(b + o_lt_row);
        d.lt_val = reinterpret_cast<float*>(b + o_lt_val);
        d.lt_part = reinterpret_cast<double*>(b + o_lt_part);
    }
    d.kev_iter = o.termination_eval_frequency >= 2 ? 2 : 1;
    for (auto& row : d.kev)
        for (auto& e : row) PDLPX_CK(cudaEventCreate(&e));
    if (d.aa_w > 0) {
        d.aa_X = reinterpret_cast<double*>(b + o_aa[0]);
        d.aa_R = reinterpret_cast<double*>(b + o_aa[1]);
        d.aa_out = reinterpret_cast<double*>(b + o_aa[2]);
        d.aa_part = reinterpret_cast<double*>(b + o_aa[3]);
        d.aa_gram = reinterpret_cast<double*>(b + o_aa[4]);
        d.aa_work = reinterpret_cast<double*>(b + o_aa[5]);
        d.aa_order = reinterpret_cast<int*>(b + o_aa[6]);
        d.aa_st = reinterpret_cast<AaState*>(b + o_aa[7]);
    }
    d.st = reinterpret_cast<DevState*>(b + o_st);
    d.dc = reinterpret_cast<DevConst*>(b + o_dc);
    d.ps = reinterpret_cast<PowerState*>(b + o_ps);

    // Upload.
    cudaStream_t s = d.stream;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        return bytes == 0 ? cudaSuccess : cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    };
    PDLPX_CK(up(d.a_ptr, sc.a.ptr.data(), 4 * (m + 1)));
    PDLPX_CK(up(d.a_idx, sc.a.idx.data(), 4 * nnz));
    PDLPX_CK(up(d.at_ptr, sc.at.ptr.data(), 4 * (n + 1)));
    PDLPX_CK(up(d.at_idx, sc.at.idx.data(), 4 * nnz));
    PDLPX_CK(up(d.a_v64, sc.a.val.data(), 8 * nnz));
    PDLPX_CK(up(d.at_v64, sc.at.val.data(), 8 * nnz));
    std::vector<float> f32;
    if (mixed) {
        toFloat(sc.a.val, f32);
        PDLPX_CK(up(d.a_v32, f32.data(), 4 * nnz));
        PDLPX_CK(cudaStreamSynchronize(s));
        toFloat(sc.at.val, f32);
        PDLPX_CK(up(d.at_v32, f32.data(), 4 * nnz));
        std::vector<ColPack<float>> cp;
        std::vector<RowPack<float>> rp;
        packCols(sc, cp);
        packRows(sc, rp);
        PDLPX_CK(up(d.cp32, cp.data(), 16 * n));
        PDLPX_CK(up(d.rp32, rp.data(), 16 * m));
        PDLPX_CK(cudaStreamSynchronize(s));
    }
    // sliced-ELL sides (each host buffer is released once its copy is done)
    auto upSell = [&](SellHost& h, int2* hdr, int* idx, double* v64, float* v32) -> cudaError_t {
        cudaError_t e;
        if ((e = up(hdr, h.hdr.data(), 8 * h.hdr.size())) != cudaSuccess) return e;
        if ((e = up(idx, h.idx.data(), 4 * h.idx.size())) != cudaSuccess) return e;
        if ((e = up(v64, h.val.data(), 8 * h.val.size())) != cudaSuccess) return e;
        if (v32 != nullptr) {
            std::vector<float> f;
            toFloat(h.val, f);
            if ((e = up(v32, f.data(), 4 * f.size())) != cudaSuccess) return e;
            if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        }
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        h = SellHost{};
        return cudaSuccess;
    };
    if (sellP) PDLPX_CK(upSell(hsP, d.sp_hdr, d.sp_idx, d.sp_v64, d.sp_v32));
    if (sellD) PDLPX_CK(upSell(hsD, d.sd_hdr, d.sd_idx, d.sd_v64, d.sd_v32));
    if (lt) {
        PDLPX_CK(up(d.lt_off, ltH.off.data(), 4 * ltH.off.size()));
        PDLPX_CK(up(d.lt_gb, ltH.gb.data(), 4 * ltH.gb.size()));
        PDLPX_CK(up(d.lt_row, ltH.row.data(), 2 * zt));
        PDLPX_CK(up(d.lt_val, ltH.val.data(), 4 * zt));
        PDLPX_CK(cudaStreamSynchronize(s));
        ltH = LongTilesHost{};
        PDLPX_CK(cudaFuncSetAttribute(primalLongTiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(tileSmemBytes(d.lt_R, d.lt_maxcols))));
    }
    {
        std::vector<ColPack<double>> cp;
        std::vector<RowPack<double>> rp;
        packCols(sc, cp);
        packRows(sc, rp);
        PDLPX_CK(up(d.cp64, cp.data(), 32 * n));
        PDLPX_CK(up(d.rp64, rp.data(), 32 * m));
        PDLPX_CK(up(d.c64, sc.c.data(), 8 * n));
        PDLPX_CK(up(d.lb64, sc.cl.data(), 8 * n));
        PDLPX_CK(up(d.ub64, sc.cu.data(), 8 * n));
        PDLPX_CK(up(d.cs64, sc.col_scale.data(), 8 * n));
        PDLPX_CK(up(d.tau64, sc.tau.data(), 8 * n));
        PDLPX_CK(up(d.rl64, sc.rl.data(), 8 * m));
        PDLPX_CK(up(d.ru64, sc.ru.data(), 8 * m));
        PDLPX_CK(up(d.rs64, sc.row_scale.data(), 8 * m));
        PDLPX_CK(up(d.sig64, sc.sigma.data(), 8 * m));
        PDLPX_CK(cudaStreamSynchronize(s));
    }
    if (o.verbose) {
        const auto tb2 = std::chrono::steady_clock::now();
        auto sec = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
            return std::chrono::duration<double>(b - a).count();
        };
        std::printf("PDLP device image: host build %.3fs (order + permute %.3fs, sliced ELL %.3fs, long tiles %.3fs), "
                    "allocation + upload %.3fs (%.1f MB)  [B200]\n",
                    sec(tb0, tb1), sec(tb0, tbp), sec(tbp, tbs), sec(tbs, tbt), sec(tb1, tb2),
                    1e-6 * static_cast<double>(d.arena_bytes));
        std::fflush(stdout);
    }
    return PDLPX_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: time the candidate launch shapes of each step kernel on the loaded
// LP (eager launches between CUDA events on the engine's stream, on a scratch
// solver state) and keep the fastest.  A candidate must beat the current pick
// by 3% to replace it, so near-ties keep the default shape.  The step kernels
// accumulate in FP64, so the pick changes results at most in the last bit of
// an FP32-stored value.  The iterates written here are overwritten by the
// solve's initialisation.
// ---------------------------------------------------------------------------
template <class T>
static int32_t autotuneShapes(DeviceLp& d, const pdlpx_options& o, bool tune_p, bool tune_d, std::string& err) {
    cudaStream_t s = d.stream;
    DevState t{};
    t.step = 1e-3;
    t.pw = 1.0;
    t.prec = precTag<T>();
    t.fpe0 = -1.0;
    *d.h_st = t;
    PDLPX_CK(cudaMemcpyAsync(d.st, d.h_st, sizeof(DevState), cudaMemcpyHostToDevice, s));
    const IterArgs<T> ia = iterArgs<T>(d, o);
    T* const xs[3] = {ia.xi, ia.xr, ia.xh};
    T* const ys[2] = {ia.yi, ia.yh};
    for (int k = 0; k < 3; ++k) PDLPX_CK(cudaMemsetAsync(xs[k], 0, sizeof(T) * static_cast<size_t>(d.n), s));
    for (int k = 0; k < 2; ++k) PDLPX_CK(cudaMemsetAsync(ys[k], 0, sizeof(T) * static_cast<size_t>(d.m), s));
    PDLPX_CK(cudaMemsetAsync(ia.xc, 0, 8 * static_cast<size_t>(d.n), s));
    PDLPX_CK(cudaMemsetAsync(ia.yc, 0, 8 * static_cast<size_t>(d.m), s));
    if (ygCopy(ia) != nullptr) PDLPX_CK(cudaMemsetAsync(ygCopy(ia), 0, sizeof(T) * static_cast<size_t>(d.m), s));
    cudaEvent_t e0, e1;
    PDLPX_CK(cudaEventCreate(&e0));
    PDLPX_CK(cudaEventCreate(&e1));
    struct G2 {
        cudaEvent_t a, b;
        ~G2() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } guard{e0, e1};
    // which: 0 primal short rows, 1 dual short rows, 2 primal long rows, 3 dual long rows
    auto timeShape = [&](int which, int shape, float& ms) -> int32_t {
        constexpr int reps = 5;
        for (int r = 0; r <= reps; ++r) {
            if (r == 1) PDLPX_CK(cudaEventRecord(e0, s));
            if (which == 0) {
                launchPrimalShort<T>(d, ia, shape, 1, s);
            } else if (which == 1) {
                launchDualShort<T>(d, ia, shape, 1, s);
            } else if (which == 2) {
                PDLPX_SHAPE_SWITCH(shape, (primalStep<GG, RR, UU, T, true><<<gridForShape(d.nlP, shape), kBlock, 0, s>>>(
                                              ia, 1, 0, d.nlP)));
            } else {
                PDLPX_SHAPE_SWITCH(shape, (dualStep<GG, RR, UU, T><<<gridForShape(d.nlD, shape), kBlock, 0, s>>>(
                                              ia, 1, 0, d.nlD)));
            }
        }
        PDLPX_CK(cudaEventRecord(e1, s));
        PDLPX_CK(cudaGetLastError());
        PDLPX_CK(cudaEventSynchronize(e1));
        PDLPX_CK(cudaEventElapsedTime(&ms, e0, e1));
        return PDLPX_OK;
    };
    for (int pass = 0; pass < 2; ++pass) {
        const bool primal = pass == 0;
        if ((primal && !tune_p) || (!primal && !tune_d)) continue;
        int& pick = primal ? d.shapeP : d.shapeD;
        const int which = primal ? 0 : 1;
        // candidates: the sliced-ELL variants where the side has them, and the
        // CSR shapes within 4x of the row-length table's lane count (the CSR
        // arrays cover the same rows in the same numbering)
        const bool has_sell = primal ? d.sp_hdr != nullptr : d.sd_hdr != nullptr;
        const int64_t rows = primal ? d.n - d.nlP : d.m - d.nlD;
        const int64_t zshort = primal ? d.nnz - d.zlP : d.nnz - d.zlD;
        const int g0 = kShapes[defaultShape(zshort, static_cast<int32_t>(rows))].G;
        float best = 0.0f;
        int32_t rc = timeShape(which, pick, best);
        if (rc != PDLPX_OK) return rc;
        for (int c = 0; c < kNumShapes + (has_sell ? kEngSell : 0); ++c) {
            if (c == pick || (!isSell(c) && (kShapes[c].G * 4 < g0 || kShapes[c].G > g0 * 4))) continue;
            float ms = 0.0f;
            rc = timeShape(which, c, ms);
            if (rc != PDLPX_OK) return rc;
            if (ms < 0.97f * best) {
                best = ms;
                pick = c;
            }
        }
    }
    // long rows (their own launches): the CSR shapes with 8 or more lanes per row
    for (int pass = 0; pass < 2; ++pass) {
        const bool primal = pass == 0;
        if ((primal && (!tune_p || d.nlP == 0)) || (!primal && (!tune_d || d.nlD == 0))) continue;
        int& pick = primal ? d.shapeLP : d.shapeLD;
        const int which = primal ? 2 : 3;
        float best = 0.0f;
        int32_t rc = timeShape(which, pick, best);
        if (rc != PDLPX_OK) return rc;
        for (int c = 0; c < kNumShapes; ++c) {
            if (c == pick || kShapes[c].G < 8) continue;
            float ms = 0.0f;
            rc = timeShape(which, c, ms);
            if (rc != PDLPX_OK) return rc;
            if (ms < 0.97f * best) {
                best = ms;
                pick = c;
            }
        }
    }
    d.tuned = true;
    return PDLPX_OK;
}

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
Engine::Engine() { pdlpx_options_default(&opt_); }
Engine::~Engine() = default;

int32_t Engine::load(int32_t m, int32_t n, int32_t nnz, const int32_t* rp, const int32_t* ci,
                     const double* v, const double* obj, const double* cl, const double* cu,
                     const double* rl, const double* ru, int32_t sense, double offset) {
    if (m < 0 || n < 0 || nnz < 0) {
        last_error = "negative dimension";
        return PDLPX_E_INVALID;
    }
    if ((n > 0 && (obj == nullptr || cl == nullptr || cu == nullptr)) ||
        (m > 0 && (rl == nullptr || ru == nullptr))) {
        last_error = "null bound / objective array";
        return PDLPX_E_INVALID;
    }
    const auto tl0 = std::chrono::steady_clock::now();
    HostLp lp;
    lp.m = m;
    lp.n = n;
    lp.maximize = sense == PDLPX_MAXIMIZE;
    if (!canonicalCsr(m, n, nnz, rp, ci, v, lp.a)) {
        last_error = "invalid CSR matrix";
        return PDLPX_E_INVALID;
    }
    lp.obj.assign(obj, obj + n);
    lp.cl.assign(cl, cl + n);
    lp.cu.assign(cu, cu + n);
    lp.rl.assign(rl, rl + m);
    lp.ru.assign(ru, ru + m);
    lp.offset = offset;
    lp_ = std::move(lp);
    loaded_ = true;
    status_ = PDLPX_STATUS_ERROR;
    objective_ = 0.0;
    iterations_ = 0;
    has_warm_ = false;
    warm_x_.clear();
    warm_y_.clear();
    x_orig_.assign(static_cast<size_t>(n), 0.0);
    y_orig_.assign(static_cast<size_t>(m), 0.0);
    const auto tl1 = std::chrono::steady_clock::now();
    rescale();
    if (opt_.verbose) {
        const auto tl2 = std::chrono::steady_clock::now();
        std::printf("PDLP load: CSR check and copy %.3fs, scaling %.3fs  [B200]\n",
                    std::chrono::duration<double>(tl1 - tl0).count(), std::chrono::duration<double>(tl2 - tl1).count());
        std::fflush(stdout);
    }
    return PDLPX_OK;
}

// Scaling pipeline; its Ruiz passes run on the device for large LPs
// (scale_on_device: 1 always, -1 from 200k nonzeros, 0 never), with identical
// results, and on the host when the device is unavailable.
void Engine::rescale() {
    std::string note;
    buildScaled(lp_, opt_, sc_, ruizFor(opt_, lp_.a.nnz(), &note));
    if (!note.empty()) last_error = note;  // the solve still runs; pdlpx_last_error says why scaling was host-side
    dev_.reset();
}

void Engine::setWarmStart(const double* x, int32_t nx, const double* y, int32_t ny) {
    warm_x_.assign(x, x + std::max(0, nx));
    warm_y_.assign(y, y + std::max(0, ny));
    has_warm_ = true;
}

void Engine::clearWarmStart() {
    warm_x_.clear();
    warm_y_.clear();
    has_warm_ = false;
}

void Engine::reducedCosts(std::vector<double>& rc) const {
    rc.assign(static_cast<size_t>(lp_.n), 0.0);
    if (!loaded_ || y_orig_.empty()) return;
    std::vector<double> aty(static_cast<size_t>(lp_.n), 0.0);
    csrMultiplyTranspose(lp_.a, y_orig_.data(), aty.data());
    for (int32_t j = 0; j < lp_.n; ++j) rc[j] = lp_.obj[j] + aty[j];
}

void Engine::addRows(int32_t rows, const int32_t* starts, const int32_t* idx, const double* vals,
                     int32_t nvals, const double* lo, const double* up) {
    if (!loaded_ || rows <= 0 || starts == nullptr) return;
    for (int32_t r = 0; r < rows; ++r) {
        const int32_t s = starts[r], e = starts[r + 1];
        if (s < 0 || e < s || e > nvals) return;
    }
    for (int32_t r = 0; r < rows; ++r) {
        std::vector<std::pair<int32_t, double>> ent;
        for (int32_t k = starts[r]; k < starts[r + 1]; ++k) ent.emplace_back(idx[k], vals[k]);
        std::stable_sort(ent.begin(), ent.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (const auto& [c, v] : ent) {  // SparseMatrix::addRow keeps entries as given (sorted)
            lp_.a.idx.push_back(c);
            lp_.a.val.push_back(v);
        }
        lp_.a.ptr.push_back(static_cast<int32_t>(lp_.a.idx.size()));
        lp_.rl.push_back(lo[r]);
        lp_.ru.push_back(up[r]);
    }
    lp_.m += rows;
    lp_.a.rows = lp_.m;
    y_orig_.resize(static_cast<size_t>(lp_.m), 0.0);
    rescale();
}

void Engine::removeRows(const int32_t* rows, int32_t count) {
    if (!loaded_ || count <= 0 || rows == nullptr) return;
    std::vector<int32_t> s(rows, rows + count);
    std::sort(s.begin(), s.end());
    s.erase(std::unique(s.begin(), s.end()), s.end());
    std::vector<char> drop(static_cast<size_t>(lp_.m), 0);
    for (int32_t r : s)
        if (r >= 0 && r < lp_.m) drop[r] = 1;
    Csr a;
    a.cols = lp_.n;
    std::vector<double> rl, ru;
    for (int32_t i = 0; i < lp_.m; ++i) {
        if (drop[i]) continue;
        for (int32_t k = lp_.a.ptr[i]; k < lp_.a.ptr[i + 1]; ++k) {
            a.idx.push_back(lp_.a.idx[k]);
            a.val.push_back(lp_.a.val[k]);
        }
        a.ptr.push_back(static_cast<int32_t>(a.idx.size()));
        rl.push_back(lp_.rl[i]);
        ru.push_back(lp_.ru[i]);
    }
    a.rows = static_cast<int32_t>(rl.size());
    lp_.a = std::move(a);
    lp_.rl = std::move(rl);
    lp_.ru = std::move(ru);
    lp_.m = lp_.a.rows;
    y_orig_.assign(static_cast<size_t>(lp_.m), 0.0);
    rescale();
}

void Engine::setColBounds(int32_t col, double lo, double up) {
    if (!loaded_ || col < 0 || col >= lp_.n) return;
    lp_.cl[col] = lo;
    lp_.cu[col] = up;
    rescale();
}

void Engine::setObjective(const double* obj, int32_t n) {
    if (!loaded_ || obj == nullptr || n != lp_.n) return;
    lp_.obj.assign(obj, obj + n);
    rescale();
}

int32_t Engine::solveTrivial(pdlpx_result* out) {
    const int32_t m = lp_.m, n = lp_.n;
    if (n == 0) {  // pdlp.cpp:813-820
        status_ = PDLPX_STATUS_OPTIMAL;
        objective_ = lp_.offset;
        iterations_ = 0;
        x_orig_.clear();
        y_orig_.assign(static_cast<size_t>(m), 0.0);
    } else {  // m == 0: bounds-only LP, pdlp.cpp:823-860
        x_orig_.resize(static_cast<size_t>(n));
        double ov = lp_.offset;
        bool unbounded = false;
        for (int32_t j = 0; j < n; ++j) {
            const double c = sc_.c[j], lb = sc_.cl[j], ub = sc_.cu[j];
            double xj;
            if (c > 0.0) {
                if (!std::isfinite(lb)) {
                    unbounded = true;
                    break;
                }
                xj = lb;
            } else if (c < 0.0) {
                if (!std::isfinite(ub)) {
                    unbounded = true;
                    break;
                }
                xj = ub;
            } else {
                xj = std::isfinite(lb) ? lb : (std::isfinite(ub) ? ub : 0.0);
            }
            x_orig_[j] = xj * sc_.col_scale[j] / sc_.con_scale;
            ov += lp_.obj[j] * x_orig_[j];
        }
        iterations_ = 0;
        if (unbounded) {
            status_ = PDLPX_STATUS_UNBOUNDED;
            objective_ = 0.0;
        } else {
            y_orig_.assign(static_cast<size_t>(m), 0.0);
            objective_ = ov;
            status_ = PDLPX_STATUS_OPTIMAL;
        }
    }
    used_gpu_ = false;
    std::memset(out, 0, sizeof(*out));
    out->status = status_;
    out->objective = objective_;
    return PDLPX_OK;
}

int32_t Engine::solve(pdlpx_result* out) {
    if (out == nullptr) {
        last_error = "null result";
        return PDLPX_E_INVALID;
    }
    if (!loaded_) {  // pdlp.cpp:802-805
        status_ = PDLPX_STATUS_ERROR;
        std::memset(out, 0, sizeof(*out));
        out->status = status_;
        last_error = "solve before load";
        return PDLPX_E_NOT_LOADED;
    }
    if (opt_.anderson_acceleration && opt_.anderson_window_size > 64) {
        last_error = "anderson_window_size above 64";
        return PDLPX_E_INVALID;
    }
    if (opt_.termination_eval_frequency <= 0) {
        last_error = "termination_eval_frequency must be positive";
        return PDLPX_E_INVALID;
    }
    if (lp_.n == 0 || lp_.m == 0) return solveTrivial(out);
    const int32_t rc = solveDevice(out);
    if (rc != PDLPX_OK) {
        status_ = PDLPX_STATUS_ERROR;
        objective_ = 0.0;
        out->status = status_;
    }
    return rc;
}

int32_t Engine::solveDevice(pdlpx_result* out) {
    std::string& err = last_error;
    const auto t0 = std::chrono::steady_clock::now();
    std::memset(out, 0, sizeof(*out));
    used_gpu_ = false;
    const bool want_mixed = wantMixed(opt_, sc_.a.rows, sc_.a.cols, sc_.a.nnz());
    const int want_aa = opt_.anderson_acceleration && opt_.anderson_window_size >= 2 ? opt_.anderson_window_size : 0;
    if (!dev_ || dev_->mixed != want_mixed || (opt_.adaptive_step != 0) != (dev_->prev_ax != nullptr) ||
        dev_->aa_w != want_aa) {
        const int32_t rc = buildDevice(dev_, sc_, opt_, err);
        if (rc != PDLPX_OK) {
            dev_.reset();
            return rc;
        }
    }
    DeviceLp& d = *dev_;
    PDLPX_CK(cudaSetDevice(d.device));
    cudaStream_t s = d.stream;
    if (opt_.autotune && !d.tuned && d.nnz >= 100000) {
        const bool tp = opt_.spmv_group_at <= 0 && opt_.shape_primal <= 0;
        const bool td = opt_.spmv_group_a <= 0 && opt_.shape_dual <= 0;
        const int32_t rc = d.mixed ? autotuneShapes<float>(d, opt_, tp, td, err)
                                   : autotuneShapes<double>(d, opt_, tp, td, err);
        if (rc != PDLPX_OK) return rc;
    }
    const int32_t m = lp_.m, n = lp_.n;
    const int N = opt_.termination_eval_frequency;
    int launches = 0;

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    PDLPX_CK(cudaEventCreate(&ev0));
    PDLPX_CK(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } ev_guard{ev0, ev1};
    PDLPX_CK(cudaEventRecord(ev0, s));

    // ---- power iteration (start vector: mt19937(42) normals, pdlp.cpp:1990-2001)
    double step = 1.0;
    {
        std::mt19937 rng(42);
        std::normal_distribution<double> dist(0.0, 1.0);
        std::vector<double> x0(static_cast<size_t>(n));
        for (auto& v : x0) v = dist(rng);
        double xn = 0.0;
        for (double v : x0) xn += v * v;
        xn = std::sqrt(xn);
        if (xn < 1e-15) xn = 1.0;
        for (auto& v : x0) v /= xn;
        toDevice(x0, d.cpos);
        PDLPX_CK(cudaMemcpyAsync(d.pi_x, x0.data(), 8 * static_cast<size_t>(n), cudaMemcpyHostToDevice, s));
        PowerState ps0{1.0, 0.0, 0.0, 0, opt_.sv_max_iter <= 0 ? 1 : 0};
        *d.h_ps = ps0;
        PDLPX_CK(cudaMemcpyAsync(d.ps, d.h_ps, sizeof(PowerState), cudaMemcpyHostToDevice, s));
        PowerArgs pa{};
        pa.x = d.pi_x;
        pa.y = d.pi_y;
        pa.xn = d.pi_xn;
        pa.part = d.pi_part;
        pa.ps = d.ps;
        pa.m = m;
        pa.n = n;
        pa.max_iter = opt_.sv_max_iter;
        pa.nb = d.nb_pi;
        pa.tol = opt_.sv_tol;
        if (!d.power) {
            // FP32 matrix values in mixed mode, FP64 in FP64 mode; vectors and sums FP64.
            cudaGraph_t g = nullptr;
            PDLPX_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            if (d.mixed) {
                const PowerMat<float> mt{d.a_ptr, d.a_idx, d.a_v32, d.at_ptr, d.at_idx, d.at_v32};
                d.launches_power = launchPowerChunk(d, pa, mt, DeviceLp::kPowerChunk);
            } else {
                const PowerMat<double> mt{d.a_ptr, d.a_idx, d.a_v64, d.at_ptr, d.at_idx, d.at_v64};
                d.launches_power = launchPowerChunk(d, pa, mt, DeviceLp::kPowerChunk);
            }
            PDLPX_CK(cudaStreamEndCapture(s, &g));
            const cudaError_t ie = cudaGraphInstantiate(&d.power, g, 0);
            cudaGraphDestroy(g);
            PDLPX_CK(ie);
        }
        for (int guard = 0; guard < 1 + opt_.sv_max_iter / DeviceLp::kPowerChunk + 1; ++guard) {
            if (d.h_ps->done) break;
            PDLPX_CK(cudaGraphLaunch(d.power, s));
            launches += d.launches_power;
            PDLPX_CK(cudaMemcpyAsync(d.h_ps, d.ps, sizeof(PowerState), cudaMemcpyDeviceToHost, s));
            PDLPX_CK(cudaStreamSynchronize(s));
        }
        const double spectral = std::sqrt(std::max(d.h_ps->s2, 1e-12));
        step = 0.998 / spectral;
    }

    // ---- constants and initial state
    DevConst dc{};
    dc.m = m;
    dc.n = n;
    dc.N = N;
    dc.max_iter = opt_.max_iter;
    dc.polish_max_iter = opt_.polish_max_iter;
    dc.linf = opt_.optimality_norm == PDLPX_NORM_LINF;
    dc.update_pw = opt_.update_primal_weight != 0;
    dc.enable_polish = opt_.enable_polishing != 0;
    dc.mixed = d.mixed;
    dc.fp64_switch = opt_.fp64_switch != 0;
    dc.adaptive = opt_.adaptive_step != 0;
    dc.precond_refresh = opt_.preconditioner_refresh != 0;
    dc.nb_rows = d.nb_rows;
    dc.nb_cols = d.nb_cols;
    dc.stall_limit = 10;
    dc.ref_fixed = opt_.reference_fixed_columns != 0;
    dc.primal_tol = opt_.primal_tol;
    dc.dual_tol = opt_.dual_tol;
    dc.opt_tol = opt_.optimality_tol;
    dc.polish_ptol = opt_.polish_primal_tol;
    dc.polish_dtol = opt_.polish_dual_tol;
    dc.kp = opt_.pid_kp;
    dc.ki = opt_.pid_ki;
    dc.kd = opt_.pid_kd;
    dc.ismooth = opt_.pid_i_smooth;
    dc.suff = opt_.restart_sufficient_decay;
    dc.nec = opt_.restart_necessary_decay;
    dc.art = opt_.restart_artificial_fraction;
    terminationNorms(lp_, opt_.optimality_norm, dc.c_norm, dc.b_norm);
    dc.obj_sign = sc_.obj_sign;
    dc.obj_scale = sc_.obj_scale;
    dc.con_scale = sc_.con_scale;
    dc.offset = lp_.offset;
    dc.step_lb = step * opt_.adaptive_step_min;
    dc.step_ub = step * opt_.adaptive_step_max;
    dc.step_down = opt_.adaptive_step_down;
    dc.step_up = opt_.adaptive_step_up;
    dc.precond_ratio = opt_.preconditioner_refresh_ratio;
    dc.switch_score = 30.0;
    dc.noise_factor = 1.0;
    PDLPX_CK(cudaMemcpyAsync(d.dc, &dc, sizeof(DevConst), cudaMemcpyHostToDevice, s));

    DevState st0{};
    st0.step = step;
    st0.pw = opt_.primal_weight;
    st0.tau_fac = static_cast<float>(step / st0.pw);
    st0.sig_fac = static_cast<float>(step * st0.pw);
    st0.prec = d.mixed ? 0 : 1;
    st0.fpe0 = -1.0;
    st0.last_fpe = std::numeric_limits<double>::infinity();
    st0.best_pw = st0.pw;
    st0.best_score = std::numeric_limits<double>::infinity();
    st0.best_kkt = std::numeric_limits<double>::infinity();
    st0.precond_pw = sc_.precond_pw;
    st0.switch_total = -1;
    *d.h_st = st0;
    PDLPX_CK(cudaMemcpyAsync(d.st, d.h_st, sizeof(DevState), cudaMemcpyHostToDevice, s));

    // ---- initial iterates (zero or warm start, pdlp.cpp:1812-1827)
    const bool warm = has_warm_ && static_cast<int32_t>(warm_x_.size()) == n &&
                      static_cast<int32_t>(warm_y_.size()) == m;
    std::vector<double> wx, wy;
    if (warm) {
        wx.resize(n);
        wy.resize(m);
        for (int32_t j = 0; j < n; ++j) wx[j] = warm_x_[j] / sc_.col_scale[j] * sc_.con_scale;
        for (int32_t i = 0; i < m; ++i) wy[i] = warm_y_[i] * sc_.obj_scale / (sc_.obj_sign * sc_.row_scale[i]);
        toDevice(wx, d.cpos);
        toDevice(wy, d.rpos);
    }
    if (d.mixed) {
        std::vector<float> fx(n, 0.0f), fy(m, 0.0f);
        if (warm) {
            for (int32_t j = 0; j < n; ++j) fx[j] = static_cast<float>(wx[j]);
            for (int32_t i = 0; i < m; ++i) fy[i] = static_cast<float>(wy[i]);
        }
        for (float* p : {d.xi32, d.xh32, d.xr32})
            PDLPX_CK(cudaMemcpyAsync(p, fx.data(), 4 * static_cast<size_t>(n), cudaMemcpyHostToDevice, s));
        for (float* p : {d.yi32, d.yh32})
            PDLPX_CK(cudaMemcpyAsync(p, fy.data(), 4 * static_cast<size_t>(m), cudaMemcpyHostToDevice, s));
        // current iterates (FP64) start equal to the FP32 anchors
        std::vector<double> dx(fx.begin(), fx.end()), dy(fy.begin(), fy.end());
        PDLPX_CK(cudaMemcpyAsync(d.xc64, dx.data(), 8 * static_cast<size_t>(n), cudaMemcpyHostToDevice, s));
        PDLPX_CK(cudaMemcpyAsync(d.yc64, dy.data(), 8 * static_cast<size_t>(m), cudaMemcpyHostToDevice, s));
        PDLPX_CK(cudaMemcpyAsync(d.yg32, fy.data(), 4 * static_cast<size_t>(m), cudaMemcpyHostToDevice, s));
        PDLPX_CK(cudaStreamSynchronize(s));
    } else {
        if (!warm) {
            wx.assign(n, 0.0);
            wy.assign(m, 0.0);
        }
        for (double* p : {d.xc64, d.xi64, d.xh64, d.xr64})
            PDLPX_CK(cudaMemcpyAsync(p, wx.data(), 8 * static_cast<size_t>(n), cudaMemcpyHostToDevice, s));
        for (double* p : {d.yc64, d.yi64, d.yh64})
            PDLPX_CK(cudaMemcpyAsync(p, wy.data(), 8 * static_cast<size_t>(m), cudaMemcpyHostToDevice, s));
        PDLPX_CK(cudaStreamSynchronize(s));
    }
    if (d.aa_st) PDLPX_CK(cudaMemsetAsync(d.aa_st, 0, sizeof(AaState), s));
    if (d.prev_ax) {
        PDLPX_CK(cudaMemsetAsync(d.prev_ax, 0, 8 * static_cast<size_t>(m), s));
        PDLPX_CK(cudaMemsetAsync(d.prev_xh, 0, 8 * static_cast<size_t>(n), s));
    }

    // ---- capture the restart-cycle graphs lazily
    auto ensureCycle = [&](int prec) -> int32_t {
        if (d.cycle[prec] && d.cycle_N[prec] == N) return PDLPX_OK;
        if (d.cycle[prec]) {
            cudaGraphExecDestroy(d.cycle[prec]);
            d.cycle[prec] = nullptr;
        }
        cudaGraph_t g = nullptr;
        PDLPX_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        d.launches_cycle[prec] = prec == 0 ? launchCycle<float>(d, opt_) : launchCycle<double>(d, opt_);
        PDLPX_CK(cudaStreamEndCapture(s, &g));
        const cudaError_t ie = cudaGraphInstantiate(&d.cycle[prec], g, 0);
        cudaGraphDestroy(g);
        PDLPX_CK(ie);
        d.cycle_N[prec] = N;
        return PDLPX_OK;
    };

    used_gpu_ = true;
    bool stopped = false;
    int switch_total = -1;
    int prec = d.mixed ? 0 : 1;
    int prev_total = 0;
    for (int p = 0; p < 2; ++p) {
        step_ms_[p][0] = step_ms_[p][1] = 0.0;
        step_samples_[p] = 0;
    }
    while (true) {
        if (timeUp(t0, opt_.max_solve_seconds)) break;
        if (stopRequested()) {
            stopped = true;
            break;
        }
        const int32_t rc = ensureCycle(prec);
        if (rc != PDLPX_OK) return rc;
        PDLPX_CK(cudaGraphLaunch(d.cycle[prec], s));
        launches += d.launches_cycle[prec];
        PDLPX_CK(cudaMemcpyAsync(d.h_st, d.st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
        PDLPX_CK(cudaStreamSynchronize(s));
        const DevState& h = *d.h_st;
        if (h.total - prev_total >= d.kev_iter) {
            // the timed iteration ran in full: read the step kernels' events of this cycle
            float a = 0.0f, b = 0.0f;
            if (cudaEventElapsedTime(&a, d.kev[prec][0], d.kev[prec][1]) == cudaSuccess &&
                cudaEventElapsedTime(&b, d.kev[prec][1], d.kev[prec][2]) == cudaSuccess) {
                step_ms_[prec][0] += a;
                step_ms_[prec][1] += b;
                ++step_samples_[prec];
            } else {
                (void)cudaGetLastError();
            }
        }
        prev_total = h.total;
        if (opt_.verbose && (h.total <= N || h.total % (10 * N) == 0)) {
            std::printf("PDLP %7d  pobj=% .8e  pinf=% .2e  dinf=% .2e  gap=% .2e  fpe=% .2e  pw=% .2e  step=% .2e  [B200%s]\n",
                        h.total, h.pobj, h.pterm, h.dterm, h.gap, h.fpe, h.pw, h.step,
                        h.prec == 0 ? " fp32" : " fp64");
            std::fflush(stdout);
        }
        if (h.done) break;
        if (h.prec != prec) {
            prec = h.prec;
            switch_total = h.total;
        }
    }
    PDLPX_CK(cudaEventRecord(ev1, s));
    PDLPX_CK(cudaEventSynchronize(ev1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);

    const DevState fin = *d.h_st;
    int32_t status;
    if (fin.done) {
        status = fin.status;
        if (status == PDLPX_STATUS_ITER_LIMIT && timeUp(t0, opt_.max_solve_seconds)) status = PDLPX_STATUS_TIME_LIMIT;
    } else if (fin.converged) {
        status = PDLPX_STATUS_OPTIMAL;  // polish interrupted (pdlp.cpp:2546-2550)
    } else {
        status = stopped ? PDLPX_STATUS_ITER_LIMIT : PDLPX_STATUS_TIME_LIMIT;
    }

    // ---- results (pdlp.cpp:2678-2712)
    const int fprec = fin.prec;
    std::vector<double> xh(n), yh(m);
    if (status == PDLPX_STATUS_OPTIMAL || status == PDLPX_STATUS_INFEASIBLE || status == PDLPX_STATUS_UNBOUNDED) {
        if (fprec == 0) {
            std::vector<float> fx(n), fy(m);
            PDLPX_CK(cudaMemcpyAsync(fx.data(), d.xh32, 4 * static_cast<size_t>(n), cudaMemcpyDeviceToHost, s));
            PDLPX_CK(cudaMemcpyAsync(fy.data(), d.yh32, 4 * static_cast<size_t>(m), cudaMemcpyDeviceToHost, s));
            PDLPX_CK(cudaStreamSynchronize(s));
            for (int32_t j = 0; j < n; ++j) xh[j] = fx[j];
            for (int32_t i = 0; i < m; ++i) yh[i] = fy[i];
        } else {
            PDLPX_CK(cudaMemcpyAsync(xh.data(), d.xh64, 8 * static_cast<size_t>(n), cudaMemcpyDeviceToHost, s));
            PDLPX_CK(cudaMemcpyAsync(yh.data(), d.yh64, 8 * static_cast<size_t>(m), cudaMemcpyDeviceToHost, s));
            PDLPX_CK(cudaStreamSynchronize(s));
        }
        fromDevice(xh, d.cpos);
        fromDevice(yh, d.rpos);
    }
    objective_ = 0.0;
    if (status == PDLPX_STATUS_OPTIMAL) {
        x_orig_.resize(n);
        const double ic = 1.0 / sc_.con_scale;
        for (int32_t j = 0; j < n; ++j) {
            double xj = xh[j] * sc_.col_scale[j] * ic;
            if (std::isfinite(lp_.cl[j])) xj = std::max(xj, lp_.cl[j]);
            if (std::isfinite(lp_.cu[j])) xj = std::min(xj, lp_.cu[j]);
            x_orig_[j] = xj;
        }
        y_orig_.resize(m);
        const double io = 1.0 / sc_.obj_scale;
        for (int32_t i = 0; i < m; ++i) y_orig_[i] = sc_.obj_sign * yh[i] * sc_.row_scale[i] * io;
        double ov = lp_.offset;
        for (int32_t j = 0; j < n; ++j) ov += lp_.obj[j] * x_orig_[j];
        objective_ = ov;
    } else if (status == PDLPX_STATUS_INFEASIBLE) {
        y_orig_.resize(m);
        const double io = 1.0 / sc_.obj_scale;
        for (int32_t i = 0; i < m; ++i) y_orig_[i] = sc_.obj_sign * yh[i] * sc_.row_scale[i] * io;
    } else if (status == PDLPX_STATUS_UNBOUNDED) {
        x_orig_.resize(n);
        const double ic = 1.0 / sc_.con_scale;
        for (int32_t j = 0; j < n; ++j) x_orig_[j] = xh[j] * sc_.col_scale[j] * ic;
    }
    status_ = status;
    iterations_ = fin.total;

    out->status = status;
    out->objective = objective_;
    out->iterations = fin.total;
    out->work_units = static_cast<double>(fin.total) *
                      (4.0 * static_cast<double>(sc_.a.nnz()) + 2.0 * static_cast<double>(m + n));
    out->rel_primal_resid = fin.pterm;
    out->rel_dual_resid = fin.dterm;
    out->rel_gap = fin.gap;
    out->primal_objective = fin.pobj;
    out->dual_objective = fin.dobj;
    out->fp64_iterations = d.mixed ? (switch_total >= 0 ? fin.total - switch_total : 0) : fin.total;
    out->restarts = fin.restarts;
    out->step_size = fin.step;
    out->primal_weight = fin.pw;
    out->solve_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    out->device_seconds = ms * 1e-3;
    out->used_gpu = 1;
    out->kernel_launches = launches;
    return PDLPX_OK;
}

// ---------------------------------------------------------------------------
// Kernel timing (roofline numerator): eager launches on the engine's stream, on
// a scratch copy of the solver state so that the step kernels of precision T
// are active; the saved state is restored afterwards.  The steps run as PDHG
// iterations (primal, dual, primal, ...) with an event between every two
// launches, so each kernel sees the cache state of the solve loop; with
// flush_bytes > 0 a write of that many bytes precedes every iteration (outside
// the timed intervals) and each iteration starts from an evicted L2.
// ---------------------------------------------------------------------------
namespace {
template <class T>
int32_t timeStepKernels(DeviceLp& d, const pdlpx_options& o, int reps, int64_t flush_bytes, double ms[3],
                        std::string& err) {
    const IterArgs<T> ia = iterArgs<T>(d, o);
    const CheckArgs<T> ca = d.check<T>(ia.xh, ia.xi, ia.yh, ia.yi);
    cudaStream_t s = d.stream;
    std::vector<cudaEvent_t> ev(3 * static_cast<size_t>(reps) + 2, nullptr);
    struct Guard {
        std::vector<cudaEvent_t>& e;
        void* flush = nullptr;
        cudaStream_t s = nullptr;
        ~Guard() {
            for (auto x : e)
                if (x) cudaEventDestroy(x);
            if (flush) cudaFreeAsync(flush, s);
        }
    } guard{ev, nullptr, s};
    for (auto& e : ev) PDLPX_CK(cudaEventCreate(&e));
    if (flush_bytes > 0) PDLPX_CK(cudaMallocAsync(&guard.flush, static_cast<size_t>(flush_bytes), s));
    // warm-up iteration; a step's time covers its long- and short-row launches
    launchPrimal<T>(d, ia, 1, s);
    launchDual<T>(d, ia, 1, s);
    for (int r = 0; r < reps; ++r) {
        if (guard.flush) PDLPX_CK(cudaMemsetAsync(guard.flush, r & 0xff, static_cast<size_t>(flush_bytes), s));
        PDLPX_CK(cudaEventRecord(ev[3 * r], s));
        launchPrimal<T>(d, ia, 1, s);
        PDLPX_CK(cudaEventRecord(ev[3 * r + 1], s));
        launchDual<T>(d, ia, 1, s);
        PDLPX_CK(cudaEventRecord(ev[3 * r + 2], s));
    }
    const size_t c0 = 3 * static_cast<size_t>(reps);
    PDLPX_CK(cudaEventRecord(ev[c0], s));
    launchChecks<T>(d, ca, s);
    PDLPX_CK(cudaEventRecord(ev[c0 + 1], s));
    PDLPX_CK(cudaGetLastError());
    PDLPX_CK(cudaEventSynchronize(ev[c0 + 1]));
    ms[0] = ms[1] = ms[2] = 0.0;
    for (int r = 0; r < reps; ++r) {
        float a = 0.0f, b = 0.0f;
        PDLPX_CK(cudaEventElapsedTime(&a, ev[3 * r], ev[3 * r + 1]));
        PDLPX_CK(cudaEventElapsedTime(&b, ev[3 * r + 1], ev[3 * r + 2]));
        ms[0] += a;
        ms[1] += b;
    }
    float c = 0.0f;
    PDLPX_CK(cudaEventElapsedTime(&c, ev[c0], ev[c0 + 1]));
    ms[0] /= reps;
    ms[1] /= reps;
    ms[2] = c;
    return PDLPX_OK;
}
}  // namespace

int32_t Engine::timeKernels(int32_t precision, int32_t reps, int64_t flush_bytes, double* ms_primal, double* ms_dual,
                            double* ms_check) {
    std::string& err = last_error;
    if (!dev_ || !used_gpu_) {
        err = "time_kernels needs a completed device solve";
        return PDLPX_E_NOT_LOADED;
    }
    if (reps <= 0) reps = 1;
    if (precision != -1 && precision != PDLPX_PREC_MIXED && precision != PDLPX_PREC_FP64) {
        err = "time_kernels: precision must be PDLPX_PREC_MIXED, PDLPX_PREC_FP64 or -1";
        return PDLPX_E_INVALID;
    }
    if (precision == PDLPX_PREC_MIXED && !dev_->mixed) {
        err = "time_kernels: the FP32 kernels need a mixed-precision solve";
        return PDLPX_E_INVALID;
    }
    DeviceLp& d = *dev_;
    PDLPX_CK(cudaSetDevice(d.device));
    cudaStream_t s = d.stream;
    DevState saved{};
    PDLPX_CK(cudaMemcpyAsync(&saved, d.st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    PDLPX_CK(cudaStreamSynchronize(s));
    DevState t = saved;
    t.done = 0;
    t.phase = 0;
    t.total = 0;
    t.inner = 0;
    if (precision != -1) t.prec = precision == PDLPX_PREC_FP64 ? 1 : 0;
    *d.h_st = t;
    PDLPX_CK(cudaMemcpyAsync(d.st, d.h_st, sizeof(DevState), cudaMemcpyHostToDevice, s));
    double ms[3] = {0, 0, 0};
    const int32_t rc = t.prec == 0 ? timeStepKernels<float>(d, opt_, reps, flush_bytes, ms, err)
                                   : timeStepKernels<double>(d, opt_, reps, flush_bytes, ms, err);
    *d.h_st = saved;
    PDLPX_CK(cudaMemcpyAsync(d.st, d.h_st, sizeof(DevState), cudaMemcpyHostToDevice, s));
    PDLPX_CK(cudaStreamSynchronize(s));
    if (rc != PDLPX_OK) return rc;
    if (ms_primal) *ms_primal = ms[0];
    if (ms_dual) *ms_dual = ms[1];
    if (ms_check) *ms_check = ms[2];
    return PDLPX_OK;
}

int32_t Engine::longTiles(int32_t* chunks, int32_t* groups) const {
    if (!dev_) return PDLPX_E_NOT_LOADED;
    if (chunks) *chunks = dev_->lt_C;
    if (groups) *groups = dev_->lt_G;
    return PDLPX_OK;
}

int32_t Engine::hotPrefix(int32_t precision, int32_t* primal, int32_t* dual) const {
    if (!dev_) return PDLPX_E_NOT_LOADED;
    const DeviceLp& d = *dev_;
    const bool fp64 = precision == PDLPX_PREC_FP64;
    if (!fp64 && !d.mixed) return PDLPX_E_INVALID;
    if (primal)
        *primal = !isSell(d.shapeP) ? 0 : fp64 ? hotPrimal<double>(d) : hotPrimal<float>(d);
    if (dual) *dual = !isSell(d.shapeD) ? 0 : fp64 ? hotDual<double>(d) : hotDual<float>(d);
    return PDLPX_OK;
}

int32_t Engine::launchConfig(int32_t* ga, int32_t* gat, int32_t* bp, int32_t* bd) const {
    if (!dev_) return PDLPX_E_NOT_LOADED;
    const DeviceLp& d = *dev_;
    if (ga) *ga = isSell(d.shapeD) ? 1 : kShapes[d.shapeD].G;
    if (gat) *gat = isSell(d.shapeP) ? 1 : kShapes[d.shapeP].G;
    if (bp) *bp = isSell(d.shapeP) ? sellGrid(d.n - d.nlP) : gridForShape(d.n - d.nlP, d.shapeP);
    if (bd) *bd = isSell(d.shapeD) ? sellGrid(d.m - d.nlD) : gridForShape(d.m - d.nlD, d.shapeD);
    return PDLPX_OK;
}

// ---------------------------------------------------------------------------
// Parity entry point: one SpMV with the engine's kernel.
// ---------------------------------------------------------------------------
int32_t deviceSpmv(int32_t rows, int32_t cols, int32_t nnz, const int32_t* rp, const int32_t* ci,
                   const double* val, const double* x, double* y, int32_t precision, int32_t group,
                   std::string& err) {
    if (rows < 0 || cols < 0 || nnz < 0 || (rows > 0 && (rp == nullptr || y == nullptr)) ||
        (nnz > 0 && (ci == nullptr || val == nullptr)) || (cols > 0 && x == nullptr)) {
        err = "invalid argument";
        return PDLPX_E_INVALID;
    }
    if (rows == 0) return PDLPX_OK;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        err = "no CUDA device visible";
        return PDLPX_E_NO_DEVICE;
    }
    const int G = group > 0 ? group : pickGroup(nnz, rows);
    const bool f64 = precision == PDLPX_PREC_FP64;
    const size_t vb = f64 ? 8 : 4;
    char* buf = nullptr;
    const size_t o_rp = 0, o_ci = o_rp + ((4 * (static_cast<size_t>(rows) + 1) + 255) & ~size_t(255)),
                 o_v = o_ci + ((4 * static_cast<size_t>(nnz) + 255) & ~size_t(255)),
                 o_x = o_v + ((vb * nnz + 255) & ~size_t(255)), o_y = o_x + ((vb * cols + 255) & ~size_t(255)),
                 total = o_y + vb * rows;
    PDLPX_CK(cudaMalloc(reinterpret_cast<void**>(&buf), total));
    struct Free {
        char* p;
        ~Free() { cudaFree(p); }
    } guard{buf};
    PDLPX_CK(cudaMemcpy(buf + o_rp, rp, 4 * (static_cast<size_t>(rows) + 1), cudaMemcpyHostToDevice));
    if (nnz > 0) PDLPX_CK(cudaMemcpy(buf + o_ci, ci, 4 * static_cast<size_t>(nnz), cudaMemcpyHostToDevice));
    const int grid = gridFor(rows, G);
    if (f64) {
        if (nnz > 0) PDLPX_CK(cudaMemcpy(buf + o_v, val, 8 * static_cast<size_t>(nnz), cudaMemcpyHostToDevice));
        if (cols > 0) PDLPX_CK(cudaMemcpy(buf + o_x, x, 8 * static_cast<size_t>(cols), cudaMemcpyHostToDevice));
        PDLPX_G_SWITCH(G, (spmvKernel<GG, double><<<grid, kBlock>>>(
                              rows, reinterpret_cast<int*>(buf + o_rp), reinterpret_cast<int*>(buf + o_ci),
                              reinterpret_cast<double*>(buf + o_v), reinterpret_cast<double*>(buf + o_x),
                              reinterpret_cast<double*>(buf + o_y))));
        PDLPX_CK(cudaGetLastError());
        PDLPX_CK(cudaMemcpy(y, buf + o_y, 8 * static_cast<size_t>(rows), cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> fv(val, val + nnz), fx(x, x + cols), fy(rows);
        if (nnz > 0) PDLPX_CK(cudaMemcpy(buf + o_v, fv.data(), 4 * static_cast<size_t>(nnz), cudaMemcpyHostToDevice));
        if (cols > 0) PDLPX_CK(cudaMemcpy(buf + o_x, fx.data(), 4 * static_cast<size_t>(cols), cudaMemcpyHostToDevice));
        PDLPX_G_SWITCH(G, (spmvKernel<GG, float><<<grid, kBlock>>>(
                              rows, reinterpret_cast<int*>(buf + o_rp), reinterpret_cast<int*>(buf + o_ci),
                              reinterpret_cast<float*>(buf + o_v), reinterpret_cast<float*>(buf + o_x),
                              reinterpret_cast<float*>(buf + o_y))));
        PDLPX_CK(cudaGetLastError());
        PDLPX_CK(cudaMemcpy(fy.data(), buf + o_y, 4 * static_cast<size_t>(rows), cudaMemcpyDeviceToHost));
        for (int32_t i = 0; i < rows; ++i) y[i] = fy[i];
    }
    return PDLPX_OK;
}

}  // namespace pdlpx
