// Packed batched PDLP (pdlpx_batch_solve).
//
// The LPs of a pack share one device image with global numbering: LP l owns
// rows [r0_l, r0_l + mp_l) and columns [c0_l, c0_l + np_l) of a block-diagonal
// A and A^T, so the gathers of the step kernels are those of the single-LP
// kernels.  Each LP's rows and columns are padded to whole tiles (a tile is as
// tall as one block of the LP's launch shape covers; padded rows and columns
// are empty, free and zero, and add nothing to any check term), and LPs with
// the same launch shape are contiguous.  A step-kernel block therefore knows
// its rows from its index alone; it loads its tile's (LP, mode) word beside
// the first matrix loads, then runs the step in the LP's current precision
// with the LP's own step size, primal weight and Halpern count.
//
// Matrix sides with short rows (mean <= 32 entries) are stored as sliced ELL:
// 32-row slices, entries column-major inside a slice and padded to the
// slice's longest row, so a warp's load of the k-th entries of its 32 rows is
// one coalesced 128-byte (FP32) request and every thread owns one row; the
// rows of each LP are renumbered longest first (stable) so a slice's rows have
// similar lengths and the heaviest tiles come first.  The renumbering is a relabelling of the LP's
// variables and constraints, undone when the results are read back.  Long
// rows keep CSR with a G-lane group per row.  The FP64 check pass and the
// power iteration read CSR.
//
// LPs restart, switch precision, polish and finish independently: per-LP
// DevState / DevConst, and the single-LP controlStep run by one warp per LP
// over the LP's tile partials in fixed order.  A restart cycle of the whole
// pack -- N iterations, the FP64 check, the controllers, restart copies, FP32
// -> FP64 hand-overs and the tile modes -- is one CUDA graph launch.  When
// finished LPs leave enough tiles idle, the host switches the launches to a
// list of the live tiles and captures a smaller graph.
//
// An LP's tiles, launch shape, storage and reduction order depend on that LP
// alone, so its result is bit-identical alone and in any mix (batch
// invariance).  A batch larger than the device budget is split into packs
// solved one after another.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <random>
#include <thread>
#include <vector>

#include "control.cuh"
#include "engine.hpp"
#include "kernels.cuh"
#include "pack.hpp"
#include "shapes.cuh"

namespace pdlpx {
namespace {

// Tile modes (the .y of a tile's info word), refreshed at the end of every cycle.
constexpr int kModeFp32 = 0, kModeFp64 = 1, kModeIdle = 2;

// Sliced-ELL launch shapes follow the kNumShapes CSR shapes: entries per lane
// per round kSellU[k], one row per thread, kBlock rows per tile.

// Rows one tile of a launch shape covers.
inline int tileRows(int shape) { return isSell(shape) ? kBlock : rowsPerBlock(shape); }
// Lanes per row of the CSR check and power kernels on that shape's tiles.
inline int checkGroup(int shape) {
    return isSell(shape) ? (kSellU[shape - kNumShapes] <= 4 ? 2 : (kSellU[shape - kNumShapes] <= 8 ? 4 : 8))
                         : kShapes[shape].G;
}

struct SellSide {
    const int2* hdr;  // per slice: first entry, entries per row (global slice = row / 32)
    const int* idx;
    const float* v32;
    const double* v64;
};

struct PackArgs {
    IterArgs<float> it32;  // global arrays of the pack (st is set per tile)
    IterArgs<double> it64;
    CheckArgs<float> ck32;
    CheckArgs<double> ck64;
    SellSide cs;         // A^T rows (primal step) of sliced-ELL shapes
    SellSide rs;         // A rows (dual step)
    int4* ctinfo;        // column tiles: (LP, mode, first column, end column)
    int4* rtinfo;        // row tiles
    const int* clist;    // live column / row tile ids after compaction
    const int* rlist;
    const int4* lpt;     // per LP: first column tile, column tiles, first row tile, row tiles
    DevState* st;
    const DevConst* dc;
    PowerState* ps;
    int* flags;           // per LP after each cycle: 1 done, 2 FP64 iterates
    int* counters;        // [0] LPs whose power iteration has finished
    double* part_cols;    // [column tile][kColSlots]
    double* part_rows;    // [row tile][kRowSlots]
    double* pi_x;         // power iteration vectors (global numbering)
    double* pi_y;
    double* pi_xn;
    double* pi_part;      // [column tile][2]
    int L, nct, nrt, mixed, sv_max_iter;
    double sv_tol;
};

constexpr int kCtlWarps = 4;  // LPs per block of the per-LP kernels

// Resident blocks per SM the CSR step kernels are compiled for: the tiles are
// latency-bound, and 5 blocks (48 registers) measured faster than 3-4 blocks
// (the compiler's own pick, 64-72 registers) and than 8 blocks with spills.
#ifndef PDLPX_PACK_MIN_BLOCKS
#define PDLPX_PACK_MIN_BLOCKS 5
#endif
// Same for the sliced-ELL step kernels: 8 blocks (32 registers) measured 28%
// faster per iteration of the 512-LP pack than 4 blocks in the FP32 phase and
// equal in the FP64 phase.
#ifndef PDLPX_SELL_MIN_BLOCKS
#define PDLPX_SELL_MIN_BLOCKS 8
#endif

__device__ __forceinline__ double combine(int op, double a, double b) {
    return op == OP_SUM ? a + b : (op == OP_MIN ? fmin(a, b) : fmax(a, b));
}

// Reduce the [tile][NS] partials of `count` tiles starting at `first` across
// one warp, in an order fixed by the tile count alone; lane 0 holds the result.
template <int NS>
__device__ __forceinline__ void warpTiles(const double* part, int first, int count, int lane, const int (&ops)[NS],
                                          double (&out)[NS]) {
#pragma unroll
    for (int s = 0; s < NS; ++s) out[s] = slotInit(ops[s]);
    for (int t = lane; t < count; t += 32) {
        const double* p = part + static_cast<size_t>(first + t) * NS;
#pragma unroll
        for (int s = 0; s < NS; ++s) out[s] = combine(ops[s], out[s], p[s]);
    }
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) out[s] = combine(ops[s], out[s], __shfl_xor_sync(0xffffffffu, out[s], off));
}

// ---- PDHG step over one CSR tile --------------------------------------------
// A launch covers the tiles [tile0, tile0 + grid) of one shape whose rows start
// at `base` (direct), or the live tiles list[list0 + b] of that shape (IND).
template <int G, int R, int U, bool IND>
__global__ void __launch_bounds__(kBlock, PDLPX_PACK_MIN_BLOCKS)
    packPrimal(PackArgs a, int tile0, int base, int list0, int koff) {
    constexpr int TR = (kBlock / G) * R;
    const int tile = IND ? a.clist[list0 + blockIdx.x] : tile0 + static_cast<int>(blockIdx.x);
    const int c0 = base + (tile - tile0) * TR;
    const int j0 = c0 + static_cast<int>(threadIdx.x) / G;
    int b[R], e[R];
    rowBounds<G, R>(a.it64.at_ptr, j0, c0 + TR, b, e);
    const int4 info = a.ctinfo[tile];
    if (info.y == kModeIdle) return;
    DevState* st = a.st + info.x;
    if (info.y == kModeFp32) {
        IterArgs<float> p = a.it32;
        p.st = st;
        primalRowsFrom<G, R, U, float>(p, j0, c0 + TR, b, e, koff);
    } else {
        IterArgs<double> p = a.it64;
        p.st = st;
        primalRowsFrom<G, R, U, double>(p, j0, c0 + TR, b, e, koff);
    }
}

template <int G, int R, int U, bool IND>
__global__ void __launch_bounds__(kBlock, PDLPX_PACK_MIN_BLOCKS)
    packDual(PackArgs a, int tile0, int base, int list0, int koff) {
    constexpr int TR = (kBlock / G) * R;
    const int tile = IND ? a.rlist[list0 + blockIdx.x] : tile0 + static_cast<int>(blockIdx.x);
    const int r0 = base + (tile - tile0) * TR;
    const int i0 = r0 + static_cast<int>(threadIdx.x) / G;
    int b[R], e[R];
    rowBounds<G, R>(a.it64.a_ptr, i0, r0 + TR, b, e);
    const int4 info = a.rtinfo[tile];
    if (info.y == kModeIdle) return;
    DevState* st = a.st + info.x;
    if (info.y == kModeFp32) {
        IterArgs<float> p = a.it32;
        p.st = st;
        dualRowsFrom<G, R, U, float>(p, i0, r0 + TR, b, e, koff);
    } else {
        IterArgs<double> p = a.it64;
        p.st = st;
        dualRowsFrom<G, R, U, double>(p, i0, r0 + TR, b, e, koff);
    }
}

// ---- PDHG step over one sliced-ELL tile (sellDot / primalSellFrom / dualSellFrom in kernels.cuh) ----
// Column j of column tile `tile` (the thread's row of the tile's slices).
template <int U>
__device__ __forceinline__ void primalSellTile(const PackArgs& a, int tile, int j, int koff) {
    const int2 h = a.cs.hdr[j / kSlice];
    const int4 info = a.ctinfo[tile];
    if (info.y == kModeIdle) return;
    DevState* st = a.st + info.x;
    if (info.y == kModeFp32) {
        IterArgs<float> p = a.it32;
        p.st = st;
        primalSellFrom<U, float>(p, a.cs.idx, a.cs.v32, j, h, koff);
    } else {
        IterArgs<double> p = a.it64;
        p.st = st;
        primalSellFrom<U, double>(p, a.cs.idx, a.cs.v64, j, h, koff);
    }
}

template <int U>
__device__ __forceinline__ void dualSellTile(const PackArgs& a, int tile, int i, int koff) {
    const int2 h = a.rs.hdr[i / kSlice];
    const int4 info = a.rtinfo[tile];
    if (info.y == kModeIdle) return;
    DevState* st = a.st + info.x;
    if (info.y == kModeFp32) {
        IterArgs<float> p = a.it32;
        p.st = st;
        dualSellFrom<U, float>(p, a.rs.idx, a.rs.v32, i, h, koff);
    } else {
        IterArgs<double> p = a.it64;
        p.st = st;
        dualSellFrom<U, double>(p, a.rs.idx, a.rs.v64, i, h, koff);
    }
}

template <int U, bool IND>
__global__ void __launch_bounds__(kBlock, PDLPX_SELL_MIN_BLOCKS) packPrimalSell(PackArgs a, int tile0, int base, int list0, int koff) {
    const int tile = IND ? a.clist[list0 + blockIdx.x] : tile0 + static_cast<int>(blockIdx.x);
    primalSellTile<U>(a, tile, base + (tile - tile0) * kBlock + static_cast<int>(threadIdx.x), koff);
}

template <int U, bool IND>
__global__ void __launch_bounds__(kBlock, PDLPX_SELL_MIN_BLOCKS) packDualSell(PackArgs a, int tile0, int base, int list0, int koff) {
    const int tile = IND ? a.rlist[list0 + blockIdx.x] : tile0 + static_cast<int>(blockIdx.x);
    dualSellTile<U>(a, tile, base + (tile - tile0) * kBlock + static_cast<int>(threadIdx.x), koff);
}

// ---- persistent restart cycle (option batch_persistent) ---------------------
// One cooperative launch runs the N PDHG iterations of a cycle over the pack's
// sliced-ELL tiles: block b takes entries b, b + grid, ... of the primal tile
// list, every block meets the others at a grid barrier, then the dual list and
// a barrier again.  Each thread's work and order are those of packPrimalSell /
// packDualSell (the same tile functions), so results are the same bits.  The
// barrier waits on a generation word with a limit on its polls; a block that
// runs out sets the error word, which the host reads after the cycle, and
// every block leaves at its next barrier.
struct PersistArgs {
    const int4* ptiles;  // (tile, first column, entries-per-round variant, 0)
    const int4* dtiles;  // (tile, first row, variant, 0)
    int np, nd, N;
    unsigned* bar;       // [0] arrivals, [1] generation
    int* err;
};
constexpr long long kBarrierPolls = 1ll << 22;  // ~0.3-1 s of 64 ns sleeps

__device__ __forceinline__ bool gridBarrier(unsigned* bar, int* err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long polls = 0;
            while (*gen == g) {
                if (++polls > kBarrierPolls) {
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *reinterpret_cast<volatile int*>(err) == 0;
}

__global__ void __launch_bounds__(kBlock, PDLPX_SELL_MIN_BLOCKS) packCycleSell(PackArgs a, PersistArgs q) {
    const int t = static_cast<int>(threadIdx.x);
    for (int k = 1; k <= q.N; ++k) {
        for (int b = static_cast<int>(blockIdx.x); b < q.np; b += static_cast<int>(gridDim.x)) {
            const int4 e = q.ptiles[b];
            if (e.z == 0)
                primalSellTile<kSellU[0]>(a, e.x, e.y + t, k);
            else
                primalSellTile<kSellU[1]>(a, e.x, e.y + t, k);
        }
        if (!gridBarrier(q.bar, q.err)) return;
        for (int b = static_cast<int>(blockIdx.x); b < q.nd; b += static_cast<int>(gridDim.x)) {
            const int4 e = q.dtiles[b];
            if (e.z == 0)
                dualSellTile<kSellU[0]>(a, e.x, e.y + t, k);
            else
                dualSellTile<kSellU[1]>(a, e.x, e.y + t, k);
        }
        if (!gridBarrier(q.bar, q.err)) return;
    }
}

// The grid barrier on its own: `rounds` barriers over a cooperative grid, with
// the words laid out as in PersistArgs (bar[0] arrivals, bar[1] generation,
// bar[2] the error word).
__global__ void barrierRounds(unsigned* bar, int rounds) {
    int* err = reinterpret_cast<int*>(bar + 2);
    for (int r = 0; r < rounds; ++r)
        if (!gridBarrier(bar, err)) return;
}

// ---- FP64 check pass, one partial per tile -----------------------------------
template <int G, bool IND>
__global__ void __launch_bounds__(kBlock) packCheckRows(PackArgs a, int tile0, int list0) {
    const int tile = IND ? a.rlist[list0 + blockIdx.x] : tile0 + static_cast<int>(blockIdx.x);
    const int4 t = a.rtinfo[tile];
    if (t.y == kModeIdle) return;
    double* out = a.part_rows + static_cast<size_t>(tile) * kRowSlots;
    constexpr int per = kBlock / G;
    if (t.y == kModeFp32)
        checkRowsRange<G, float>(a.ck32, a.dc[t.x], t.z, t.w, per, out);
    else
        checkRowsRange<G, double>(a.ck64, a.dc[t.x], t.z, t.w, per, out);
}

template <int G, bool IND>
__global__ void __launch_bounds__(kBlock) packCheckCols(PackArgs a, int tile0, int list0) {
    const int tile = IND ? a.clist[list0 + blockIdx.x] : tile0 + static_cast<int>(blockIdx.x);
    const int4 t = a.ctinfo[tile];
    if (t.y == kModeIdle) return;
    double* out = a.part_cols + static_cast<size_t>(tile) * kColSlots;
    constexpr int per = kBlock / G;
    if (t.y == kModeFp32)
        checkColsRange<G, float>(a.ck32, a.dc[t.x], t.z, t.w, per, out);
    else
        checkColsRange<G, double>(a.ck64, a.dc[t.x], t.z, t.w, per, out);
}

// ---- per-LP controller: one warp per LP ---------------------------------------
__global__ void __launch_bounds__(32 * kCtlWarps) packController(PackArgs a) {
    const int l = blockIdx.x * kCtlWarps + static_cast<int>(threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (l >= a.L) return;
    DevState* st = a.st + l;
    if (st->done) return;
    const int4 t = a.lpt[l];
    int rops[kRowSlots], cops[kColSlots];
#pragma unroll
    for (int s = 0; s < kRowSlots; ++s) rops[s] = rowSlotOp(s);
#pragma unroll
    for (int s = 0; s < kColSlots; ++s) cops[s] = colSlotOp(s);
    double rows[kRowSlots], cols[kColSlots];
    warpTiles<kRowSlots>(a.part_rows, t.z, t.w, lane, rops, rows);
    warpTiles<kColSlots>(a.part_cols, t.x, t.y, lane, cops, cols);
    if (lane == 0) {
        DevState s = *st;
        controlStep(s, a.dc[l], rows, cols);
        *st = s;
    }
}

// Restart copy (pdlp_kernels.cu:377-405) and FP32 -> FP64 hand-over per tile:
// blocks [0, ncol) take column tiles, the rest row tiles (lists after compaction).
__global__ void __launch_bounds__(kBlock) packRestart(PackArgs a, int ncol, int use_list) {
    const bool col = static_cast<int>(blockIdx.x) < ncol;
    const int k = col ? static_cast<int>(blockIdx.x) : static_cast<int>(blockIdx.x) - ncol;
    const int tile = use_list ? (col ? a.clist[k] : a.rlist[k]) : k;
    const int4 t = col ? a.ctinfo[tile] : a.rtinfo[tile];
    if (t.y == kModeIdle) return;
    const DevState* st = a.st + t.x;
    if (st->done) return;
    const int prec = st->prec;
    const bool restart = st->restart != 0;
    const bool promote = prec == 0 && st->promote != 0;
    if (!restart && !promote) return;
    for (int q = t.z + threadIdx.x; q < t.w; q += kBlock) {
        if (col) {
            if (prec == 0) {
                if (restart) {
                    const float v = a.it32.xh[q];
                    a.it32.xi[q] = v;
                    a.it32.xc[q] = v;
                }
                if (promote) {
                    a.it64.xi[q] = a.it32.xi[q];
                    a.it64.xh[q] = a.it32.xh[q];
                }
            } else {
                const double v = a.it64.xh[q];
                a.it64.xi[q] = v;
                a.it64.xc[q] = v;
            }
        } else {
            if (prec == 0) {
                if (restart) {
                    const float v = a.it32.yh[q];
                    a.it32.yi[q] = v;
                    a.it32.yc[q] = v;
                }
                if (promote) {
                    a.it64.yi[q] = a.it32.yi[q];
                    a.it64.yh[q] = a.it32.yh[q];
                }
            } else {
                const double v = a.it64.yh[q];
                a.it64.yi[q] = v;
                a.it64.yc[q] = v;
            }
        }
    }
}

// Hand-over bookkeeping and the per-LP flags the host reads after a cycle.
__global__ void packFinish(PackArgs a) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= a.L) return;
    DevState* st = a.st + l;
    if (!st->done && st->prec == 0 && st->promote) {
        st->prec = 1;
        st->switch_total = st->total;
    }
    a.flags[l] = (st->done ? 1 : 0) | (st->prec ? 2 : 0);
}

// Mode of every tile for the next cycle: idle once its LP is done, else its precision.
__global__ void packModes(PackArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nct + a.nrt) return;
    int4* info = k < a.nct ? a.ctinfo + k : a.rtinfo + (k - a.nct);
    const DevState* st = a.st + info->x;
    info->y = st->done ? kModeIdle : (st->prec ? kModeFp64 : kModeFp32);
}

// ---- power iteration on A^T A per LP (pdlp.cpp:748-795, 1985-2041) ---------------
template <int G>
__global__ void __launch_bounds__(kBlock) packPowerA(PackArgs a, int tile0) {
    const int4 t = a.rtinfo[tile0 + blockIdx.x];
    if (a.ps[t.x].done) return;
    constexpr int per = kBlock / G;
    const int lane = threadIdx.x % G;
    for (int base = t.z; base < t.w; base += per) {
        const int i = base + threadIdx.x / G;
        const bool valid = i < t.w;
        double s = 0.0;
        if (valid) {
            const int b = a.it64.a_ptr[i], e = a.it64.a_ptr[i + 1];
            s = a.mixed ? rowDot<G, double>(b, e, lane, a.it32.a_idx, a.it32.a_val, a.pi_x)
                        : rowDot<G, double>(b, e, lane, a.it64.a_idx, a.it64.a_val, a.pi_x);
        }
        s = groupSum<G>(s);
        if (valid && lane == 0) a.pi_y[i] = s;
    }
}

template <int G>
__global__ void __launch_bounds__(kBlock) packPowerAt(PackArgs a, int tile0) {
    const int tile = tile0 + blockIdx.x;
    const int4 t = a.ctinfo[tile];
    if (a.ps[t.x].done) return;
    constexpr int per = kBlock / G;
    const int lane = threadIdx.x % G;
    double acc[2] = {0.0, 0.0};
    for (int base = t.z; base < t.w; base += per) {
        const int j = base + threadIdx.x / G;
        const bool valid = j < t.w;
        double s = 0.0;
        if (valid) {
            const int b = a.it64.at_ptr[j], e = a.it64.at_ptr[j + 1];
            s = a.mixed ? rowDot<G, double>(b, e, lane, a.it32.at_idx, a.it32.at_val, a.pi_y)
                        : rowDot<G, double>(b, e, lane, a.it64.at_idx, a.it64.at_val, a.pi_y);
        }
        s = groupSum<G>(s);
        if (valid && lane == 0) {
            a.pi_xn[j] = s;
            acc[0] += a.pi_x[j] * s;
            acc[1] += s * s;
        }
    }
    const int ops[2] = {OP_SUM, OP_SUM};
    blockReduceSlots<2>(acc, ops, a.pi_part + static_cast<size_t>(tile) * 2);
}

__global__ void __launch_bounds__(32 * kCtlWarps) packPowerFinish1(PackArgs a) {
    const int l = blockIdx.x * kCtlWarps + static_cast<int>(threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (l >= a.L || a.ps[l].done) return;
    const int4 t = a.lpt[l];
    const int ops[2] = {OP_SUM, OP_SUM};
    double out[2];
    warpTiles<2>(a.pi_part, t.x, t.y, lane, ops, out);
    if (lane == 0) {
        a.ps[l].s2 = out[0];
        a.ps[l].nrm = sqrt(out[1]);
    }
}

__global__ void __launch_bounds__(kBlock) packPowerNormalize(PackArgs a) {
    const int tile = blockIdx.x;
    const int4 t = a.ctinfo[tile];
    const PowerState& ps = a.ps[t.x];
    if (ps.done) return;
    const double s2 = ps.s2, nrm = ps.nrm;
    double acc[1] = {0.0};
    for (int j = t.z + threadIdx.x; j < t.w; j += kBlock) {
        const double xn = a.pi_xn[j];
        const double d = xn - s2 * a.pi_x[j];
        acc[0] += d * d;
        if (nrm >= 1e-15) a.pi_x[j] = xn / nrm;
    }
    const int ops[1] = {OP_SUM};
    blockReduceSlots<1>(acc, ops, a.pi_part + static_cast<size_t>(tile) * 2);
}

__global__ void __launch_bounds__(32 * kCtlWarps) packPowerFinish2(PackArgs a) {
    const int l = blockIdx.x * kCtlWarps + static_cast<int>(threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (l >= a.L || a.ps[l].done) return;
    const int4 t = a.lpt[l];
    double acc = 0.0;
    for (int k = lane; k < t.y; k += 32) acc += a.pi_part[static_cast<size_t>(t.x + k) * 2];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) {
        PowerState& p = a.ps[l];
        p.resid = sqrt(acc);
        p.iter += 1;
        if (p.nrm < 1e-15 || p.resid < a.sv_tol * fabs(p.s2) || p.iter >= a.sv_max_iter) {
            p.done = 1;
            atomicAdd(a.counters, 1);
        }
    }
}

// Step size from the spectral-norm estimate (0.998 / ||A||_2, pdlp.cpp:796-800).
__global__ void packInitStep(PackArgs a) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= a.L) return;
    DevState& s = a.st[l];
    const double step = 0.998 / sqrt(fmax(a.ps[l].s2, 1e-12));
    s.step = step;
    s.tau_fac = static_cast<float>(step / s.pw);
    s.sig_fac = static_cast<float>(step * s.pw);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

// One side of an LP in its pack numbering: new position -> original row
// (order), original row -> new position (pos), and for sliced-ELL sides the
// per-slice row lengths.
struct SideOrder {
    std::vector<int32_t> order, pos;
    std::vector<int32_t> slice_len;
    int64_t entries = 0;  // sliced-ELL entries (padded)
};

// Renumbering of `rows` CSR rows padded to `padded`: identity for CSR sides;
// for sliced-ELL sides, rows sorted by length over the whole LP (longest
// first, stable), then the slice lengths.  (Sorting inside each 256-row tile
// only measured 2.91 s against 2.84 s for the 512-LP workload on B200: the
// whole-LP order puts the heaviest tiles first.)
void orderSide(const std::vector<int32_t>& ptr, int32_t rows, int64_t padded, bool sell, SideOrder& so) {
    so.order.resize(rows);
    std::iota(so.order.begin(), so.order.end(), 0);
    if (sell) {
        std::stable_sort(so.order.begin(), so.order.end(), [&](int32_t a, int32_t b) {
            return ptr[a + 1] - ptr[a] > ptr[b + 1] - ptr[b];
        });
        const int64_t slices = padded / kSlice;
        so.slice_len.assign(slices, 0);
        so.entries = 0;
        for (int64_t s = 0; s < slices; ++s) {
            int32_t len = 0;
            for (int64_t r = s * kSlice; r < std::min<int64_t>(rows, (s + 1) * kSlice); ++r)
                len = std::max(len, ptr[so.order[r] + 1] - ptr[so.order[r]]);
            so.slice_len[s] = len;
            so.entries += static_cast<int64_t>(len) * kSlice;
        }
    }
    so.pos.resize(rows);
    for (int32_t k = 0; k < rows; ++k) so.pos[so.order[k]] = k;
}

struct Item {
    HostLp lp;
    std::vector<double> warm_x, warm_y;  // warm start in original space (both or neither)
    ScaledLp sc;
    bool trivial = false;
    int shapeP = 0, shapeD = 0;
    int nct = 0, nrt = 0;      // tiles
    int64_t np = 0, mp = 0;    // columns / rows padded to whole tiles
    SideOrder cols, rows;      // renumbering of columns (A^T rows) and rows
    size_t bytes = 0;          // share of a pack's device image
    std::string scale_note;    // why the device Ruiz passes fell back to the host (empty: they did not)
    // position within its pack
    int64_t r0 = 0, c0 = 0;    // first row, first column
    int64_t za = 0, zt = 0;    // first entry of A / of A^T
    int64_t ec = 0, er = 0;    // first sliced-ELL entry of A^T / of A
    int ct0 = 0, rt0 = 0;      // first column tile, first row tile
    int l = 0;
};

size_t al256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

// Device bytes an LP adds to a pack (image + scratch), for the pack split.
size_t itemBytes(const Item& it, bool mixed) {
    const size_t m = it.mp, n = it.np, z = it.sc.a.nnz();
    size_t b = 4 * (m + n) + z * (8 + 16 + (mixed ? 8 : 0));           // pointers, indices, values
    b += n * (32 + 40 + 8 + 24 + 24) + m * (32 + 32 + 8 + 16 + 8);     // packs, checks, FP64 iterates, power
    if (mixed) b += n * (16 + 12) + m * (16 + 8);
    b += static_cast<size_t>(it.cols.entries + it.rows.entries) * (4 + 8 + (mixed ? 4 : 0)) + (m + n) / 4;
    b += static_cast<size_t>(it.nct) * (16 + 4 + 8 * kColSlots + 16) + static_cast<size_t>(it.nrt) * (16 + 4 + 8 * kRowSlots);
    b += sizeof(DevState) + sizeof(DevConst) + sizeof(PowerState) + 32;
    return b;
}

template <class F>
void parallelFor(int count, F&& f) {
    const int hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const int nt = std::min(hw, std::max(1, count));
    if (nt <= 1) {
        for (int k = 0; k < count; ++k) f(k);
        return;
    }
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

// Host wait for the work queued on a stream, sleeping instead of spinning: a
// restart cycle runs for milliseconds, and the host cores are wanted by the
// request server's preparation threads meanwhile.
struct SleepWait {
    cudaEvent_t ev = nullptr;
    ~SleepWait() {
        if (ev) cudaEventDestroy(ev);
    }
    cudaError_t wait(cudaStream_t s) {
        cudaError_t e = cudaSuccess;
        if (!ev) e = cudaEventCreateWithFlags(&ev, cudaEventBlockingSync | cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(ev, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev);
        return e;
    }
};

// One launch of a step / check kernel: the tiles of one shape class, all of them
// (list0 < 0: tiles [tile0, tile0 + count) from row `base`) or `count` live ones
// listed from list0.
// `kern` is the shape whose kernel runs the class: the class's own shape, or
// for a sliced-ELL class the entries-per-round variant the pack's autotuner
// picked (all variants read the same slices and sum every row in entry order).
struct Launch {
    int shape, tile0, base, count, list0;
    int kern = -1;
    int k() const { return kern >= 0 ? kern : shape; }
};

// Shapes in placement order: sliced-ELL classes first (their rows start at 0
// and stay aligned to whole slices), then the CSR classes.
std::vector<int> placementOrder() {
    std::vector<int> v;
    for (int s = 0; s < kNumSell; ++s) v.push_back(kNumShapes + s);
    for (int s = 0; s < kNumShapes; ++s) v.push_back(s);
    return v;
}

// Device image and graphs of one pack.
struct Pack {
    std::vector<Item*> items;
    bool mixed = true;
    int L = 0;
    int64_t M = 0, Nc = 0, Z = 0;  // padded rows, padded columns, entries
    int64_t Ec = 0, Er = 0;        // sliced-ELL entries of A^T / A
    int64_t Sc = 0, Sr = 0;        // slices (sliced-ELL prefix of the columns / rows, / 32)
    int nct = 0, nrt = 0;          // all tiles
    // arena layout
    size_t o_aptr, o_aidx, o_atptr, o_atidx, o_av32, o_atv32, o_av64, o_atv64, o_cp32, o_rp32, o_cp64, o_rp64;
    size_t o_chdr, o_cidx, o_cv32, o_cv64, o_rhdr, o_ridx, o_rv32, o_rv64;
    size_t o_c, o_lb, o_ub, o_cs, o_tau, o_rl, o_ru, o_rs, o_sig;
    size_t o_st, o_dc, o_ps, o_ctinfo, o_rtinfo, o_lpt;
    size_t image_end;  // [0, image_end) is uploaded from the host image
    size_t o_xc, o_xi32, o_xr32, o_xh32, o_xi64, o_xr64, o_xh64, o_yc, o_yi32, o_yh32, o_yi64, o_yh64;
    size_t iter_end;   // [image_end, iter_end): iterates (zero or warm start)
    size_t o_pix, o_piy, o_pixn, o_pipart, o_pcols, o_prows, o_clist, o_rlist, o_flags, o_counters;
    size_t total;
    char* d = nullptr;
    cudaStream_t s = nullptr;
    cudaGraphExec_t cycle = nullptr, power = nullptr;
    int cycle_launches = 0, power_launches = 0;
    std::vector<Launch> cls_c, cls_r;  // every tile, per shape class
    std::vector<Launch> lc, lr;        // launches of the current cycle graph
    bool listed = false;               // lc / lr run over the live-tile lists
    int live_ct = 0, live_rt = 0;      // tiles in the current launches
    std::vector<int> h_cl, h_rl;       // host copies of the live-tile lists
    PackArgs args{};
    // persistent cycle (option batch_persistent): tile lists, barrier words
    // [arrivals, generation, error, -], cooperative grid
    bool persist = false;
    int persist_grid = 0;
    char* pd = nullptr;
    std::vector<int4> h_ptiles, h_dtiles;

    // Stream-ordered allocation: packs of a request server come and go while
    // other packs run, and a plain free would wait for the whole device.
    ~Pack() {
        if (cycle) cudaGraphExecDestroy(cycle);
        if (power) cudaGraphExecDestroy(power);
        if (pd) cudaFreeAsync(pd, s);
        if (d) cudaFreeAsync(d, s);
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }

    // Positions: columns grouped by primal shape, rows by dual shape, LP order
    // within a shape; each LP padded to whole tiles.
    void place() {
        for (int side = 0; side < 2; ++side) {
            int64_t pos = 0, z = 0, ent = 0, sell_rows = 0;
            int tiles = 0;
            std::vector<Launch>& cls = side == 0 ? cls_c : cls_r;
            for (int shape : placementOrder()) {
                Launch c{shape, tiles, static_cast<int>(pos), 0, -1};
                for (Item* it : items) {
                    if ((side == 0 ? it->shapeP : it->shapeD) != shape) continue;
                    if (side == 0) {
                        it->c0 = pos;
                        it->zt = z;
                        it->ec = ent;
                        it->ct0 = tiles;
                        pos += it->np;
                        tiles += it->nct;
                        ent += it->cols.entries;
                    } else {
                        it->r0 = pos;
                        it->za = z;
                        it->er = ent;
                        it->rt0 = tiles;
                        pos += it->mp;
                        tiles += it->nrt;
                        ent += it->rows.entries;
                    }
                    z += it->sc.a.nnz();
                }
                if (isSell(shape)) sell_rows = pos;
                c.count = tiles - c.tile0;
                if (c.count > 0) cls.push_back(c);
            }
            if (side == 0) {
                Nc = pos;
                nct = tiles;
                Z = z;
                Ec = ent;
                Sc = sell_rows / kSlice;
            } else {
                M = pos;
                nrt = tiles;
                Er = ent;
                Sr = sell_rows / kSlice;
            }
        }
        lc = cls_c;
        lr = cls_r;
        listed = false;
        live_ct = nct;
        live_rt = nrt;
    }

    void layout() {
        size_t o = 0;
        auto take = [&](size_t b) {
            const size_t at = o;
            o += al256(b);
            return at;
        };
        const size_t m = M, n = Nc, z = Z;
        o_aptr = take(4 * (m + 1));
        o_aidx = take(4 * z);
        o_atptr = take(4 * (n + 1));
        o_atidx = take(4 * z);
        o_av32 = mixed ? take(4 * z) : 0;
        o_atv32 = mixed ? take(4 * z) : 0;
        o_av64 = take(8 * z);
        o_atv64 = take(8 * z);
        o_chdr = take(8 * static_cast<size_t>(std::max<int64_t>(Sc, 1)));
        o_cidx = take(4 * static_cast<size_t>(Ec));
        o_cv32 = mixed ? take(4 * static_cast<size_t>(Ec)) : 0;
        o_cv64 = take(8 * static_cast<size_t>(Ec));
        o_rhdr = take(8 * static_cast<size_t>(std::max<int64_t>(Sr, 1)));
        o_ridx = take(4 * static_cast<size_t>(Er));
        o_rv32 = mixed ? take(4 * static_cast<size_t>(Er)) : 0;
        o_rv64 = take(8 * static_cast<size_t>(Er));
        o_cp32 = mixed ? take(16 * n) : 0;
        o_rp32 = mixed ? take(16 * m) : 0;
        o_cp64 = take(32 * n);
        o_rp64 = take(32 * m);
        o_c = take(8 * n);
        o_lb = take(8 * n);
        o_ub = take(8 * n);
        o_cs = take(8 * n);
        o_tau = take(8 * n);
        o_rl = take(8 * m);
        o_ru = take(8 * m);
        o_rs = take(8 * m);
        o_sig = take(8 * m);
        o_st = take(sizeof(DevState) * L);
        o_dc = take(sizeof(DevConst) * L);
        o_ps = take(sizeof(PowerState) * L);
        o_ctinfo = take(sizeof(int4) * nct);
        o_rtinfo = take(sizeof(int4) * nrt);
        o_lpt = take(sizeof(int4) * L);
        o_pix = take(8 * n);
        image_end = o;
        o_xc = take(8 * n);
        o_xi32 = mixed ? take(4 * n) : 0;
        o_xr32 = mixed ? take(4 * n) : 0;
        o_xh32 = mixed ? take(4 * n) : 0;
        o_xi64 = take(8 * n);
        o_xr64 = take(8 * n);
        o_xh64 = take(8 * n);
        o_yc = take(8 * m);
        o_yi32 = mixed ? take(4 * m) : 0;
        o_yh32 = mixed ? take(4 * m) : 0;
        o_yi64 = take(8 * m);
        o_yh64 = take(8 * m);
        iter_end = o;
        o_piy = take(8 * m);
        o_pixn = take(8 * n);
        o_pipart = take(16 * static_cast<size_t>(nct));
        o_pcols = take(8 * kColSlots * static_cast<size_t>(nct));
        o_prows = take(8 * kRowSlots * static_cast<size_t>(nrt));
        o_clist = take(4 * static_cast<size_t>(nct));
        o_rlist = take(4 * static_cast<size_t>(nrt));
        o_flags = take(4 * static_cast<size_t>(L));
        o_counters = take(64);
        total = o;
    }

    template <class T>
    T* P(size_t off) const {
        return reinterpret_cast<T*>(d + off);
    }

    void makeArgs(const pdlpx_options& o) {
        PackArgs& a = args;
        auto fillIter = [&](auto& it, auto* av, auto* atv, auto* cp, auto* rp, auto* xi, auto* xr, auto* xh, auto* yi,
                            auto* yh) {
            it.at_ptr = P<int>(o_atptr);
            it.at_idx = P<int>(o_atidx);
            it.at_val = atv;
            it.a_ptr = P<int>(o_aptr);
            it.a_idx = P<int>(o_aidx);
            it.a_val = av;
            it.cp = cp;
            it.rp = rp;
            it.xc = P<double>(o_xc);
            it.xi = xi;
            it.xr = xr;
            it.xh = xh;
            it.yc = P<double>(o_yc);
            it.yi = yi;
            it.yh = yh;
            it.st = nullptr;
            it.m = static_cast<int>(M);
            it.n = static_cast<int>(Nc);
            it.max_iter = o.max_iter;
            it.polish_max_iter = o.polish_max_iter;
            it.N = o.termination_eval_frequency;
        };
        fillIter(a.it64, P<double>(o_av64), P<double>(o_atv64), P<ColPack<double>>(o_cp64), P<RowPack<double>>(o_rp64),
                 P<double>(o_xi64), P<double>(o_xr64), P<double>(o_xh64), P<double>(o_yi64), P<double>(o_yh64));
        if (mixed)
            fillIter(a.it32, P<float>(o_av32), P<float>(o_atv32), P<ColPack<float>>(o_cp32), P<RowPack<float>>(o_rp32),
                     P<float>(o_xi32), P<float>(o_xr32), P<float>(o_xh32), P<float>(o_yi32), P<float>(o_yh32));
        auto fillCheck = [&](auto& c, const auto& it) {
            c.a_ptr = P<int>(o_aptr);
            c.a_idx = P<int>(o_aidx);
            c.a_val = P<double>(o_av64);
            c.at_ptr = P<int>(o_atptr);
            c.at_idx = P<int>(o_atidx);
            c.at_val = P<double>(o_atv64);
            c.xh = it.xh;
            c.xi = it.xi;
            c.yh = it.yh;
            c.yi = it.yi;
            c.c64 = P<double>(o_c);
            c.lb64 = P<double>(o_lb);
            c.ub64 = P<double>(o_ub);
            c.cs64 = P<double>(o_cs);
            c.tau64 = P<double>(o_tau);
            c.rl64 = P<double>(o_rl);
            c.ru64 = P<double>(o_ru);
            c.rs64 = P<double>(o_rs);
            c.sig64 = P<double>(o_sig);
            c.prev_ax = nullptr;
            c.prev_xh = nullptr;
            c.part_rows = P<double>(o_prows);
            c.part_cols = P<double>(o_pcols);
            c.dc = nullptr;
            c.st = nullptr;
            c.m = static_cast<int>(M);
            c.n = static_cast<int>(Nc);
        };
        fillCheck(a.ck64, a.it64);
        if (mixed) fillCheck(a.ck32, a.it32);
        a.cs = SellSide{P<int2>(o_chdr), P<int>(o_cidx), mixed ? P<float>(o_cv32) : nullptr, P<double>(o_cv64)};
        a.rs = SellSide{P<int2>(o_rhdr), P<int>(o_ridx), mixed ? P<float>(o_rv32) : nullptr, P<double>(o_rv64)};
        a.ctinfo = P<int4>(o_ctinfo);
        a.rtinfo = P<int4>(o_rtinfo);
        a.clist = P<int>(o_clist);
        a.rlist = P<int>(o_rlist);
        a.lpt = P<int4>(o_lpt);
        a.st = P<DevState>(o_st);
        a.dc = P<DevConst>(o_dc);
        a.ps = P<PowerState>(o_ps);
        a.flags = P<int>(o_flags);
        a.counters = P<int>(o_counters);
        a.part_cols = P<double>(o_pcols);
        a.part_rows = P<double>(o_prows);
        a.pi_x = P<double>(o_pix);
        a.pi_y = P<double>(o_piy);
        a.pi_xn = P<double>(o_pixn);
        a.pi_part = P<double>(o_pipart);
        a.L = L;
        a.nct = nct;
        a.nrt = nrt;
        a.mixed = mixed ? 1 : 0;
        a.sv_max_iter = o.sv_max_iter;
        a.sv_tol = o.sv_tol;
    }

    // Live-tile lists of the LPs with keep[l] set (shape class by shape class,
    // tile order kept) and the launches over them.
    void liveLists(const std::vector<char>& keep, std::vector<int>& cl, std::vector<int>& rl) {
        cl.clear();
        rl.clear();
        lc.clear();
        lr.clear();
        for (int side = 0; side < 2; ++side) {
            std::vector<int>& out = side == 0 ? cl : rl;
            for (const Launch& c : side == 0 ? cls_c : cls_r) {
                const int list0 = static_cast<int>(out.size());
                for (const Item* it : items) {
                    if (!keep[it->l] || (side == 0 ? it->shapeP : it->shapeD) != c.shape) continue;
                    const int first = side == 0 ? it->ct0 : it->rt0;
                    const int count = side == 0 ? it->nct : it->nrt;
                    for (int k = 0; k < count; ++k) out.push_back(first + k);
                }
                const int count = static_cast<int>(out.size()) - list0;
                if (count > 0) (side == 0 ? lc : lr).push_back(Launch{c.shape, c.tile0, c.base, count, list0, c.kern});
            }
        }
        listed = true;
        live_ct = static_cast<int>(cl.size());
        live_rt = static_cast<int>(rl.size());
        h_cl = cl;
        h_rl = rl;
    }

    // Whether the current launches can run as one persistent cycle: every
    // class sliced ELL with 4 or 8 entries per round.
    bool persistable() const {
        for (const auto* v : {&lc, &lr})
            for (const Launch& c : *v)
                if (!isSell(c.shape) || c.k() - kNumShapes > 1) return false;
        return true;
    }

    // Tile lists of the persistent cycle for the current launches (the same
    // tiles and first rows the per-class launches cover), uploaded on the
    // pack's stream.
    cudaError_t uploadPersistTiles() {
        h_ptiles.clear();
        h_dtiles.clear();
        for (int side = 0; side < 2; ++side) {
            std::vector<int4>& out = side == 0 ? h_ptiles : h_dtiles;
            const std::vector<int>& list = side == 0 ? h_cl : h_rl;
            for (const Launch& c : side == 0 ? lc : lr)
                for (int b = 0; b < c.count; ++b) {
                    const int tile = listed ? list[c.list0 + b] : c.tile0 + b;
                    out.push_back(make_int4(tile, c.base + (tile - c.tile0) * kBlock, c.k() - kNumShapes, 0));
                }
        }
        cudaError_t e = cudaSuccess;
        if (!h_ptiles.empty())
            e = cudaMemcpyAsync(pd + 16, h_ptiles.data(), sizeof(int4) * h_ptiles.size(), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && !h_dtiles.empty())
            e = cudaMemcpyAsync(pd + 16 + sizeof(int4) * static_cast<size_t>(nct), h_dtiles.data(),
                                sizeof(int4) * h_dtiles.size(), cudaMemcpyHostToDevice, s);
        return e;
    }

    // One persistent cycle of N iterations (barrier words cleared first).
    cudaError_t launchPersistent(int N) {
        PersistArgs q{reinterpret_cast<const int4*>(pd + 16),
                      reinterpret_cast<const int4*>(pd + 16 + sizeof(int4) * static_cast<size_t>(nct)),
                      static_cast<int>(h_ptiles.size()), static_cast<int>(h_dtiles.size()), N,
                      reinterpret_cast<unsigned*>(pd), reinterpret_cast<int*>(pd + 8)};
        cudaError_t e = cudaMemsetAsync(pd, 0, 16, s);
        if (e != cudaSuccess) return e;
        void* kargs[] = {&args, &q};
        return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&packCycleSell), dim3(persist_grid),
                                           dim3(kBlock), kargs, 0, s);
    }

    void launchPrimal(const Launch& c, int k) {
        const PackArgs& a = args;
        if (isSell(c.shape)) {
            if (listed) {
                PDLPX_SELL_SWITCH(c.k(), (packPrimalSell<UU, true><<<c.count, kBlock, 0, s>>>(a, c.tile0, c.base, c.list0, k)));
            } else {
                PDLPX_SELL_SWITCH(c.k(), (packPrimalSell<UU, false><<<c.count, kBlock, 0, s>>>(a, c.tile0, c.base, 0, k)));
            }
        } else if (listed) {
            PDLPX_SHAPE_SWITCH(c.shape, (packPrimal<GG, RR, UU, true><<<c.count, kBlock, 0, s>>>(a, c.tile0, c.base, c.list0, k)));
        } else {
            PDLPX_SHAPE_SWITCH(c.shape, (packPrimal<GG, RR, UU, false><<<c.count, kBlock, 0, s>>>(a, c.tile0, c.base, 0, k)));
        }
    }

    void launchDual(const Launch& c, int k) {
        const PackArgs& a = args;
        if (isSell(c.shape)) {
            if (listed) {
                PDLPX_SELL_SWITCH(c.k(), (packDualSell<UU, true><<<c.count, kBlock, 0, s>>>(a, c.tile0, c.base, c.list0, k)));
            } else {
                PDLPX_SELL_SWITCH(c.k(), (packDualSell<UU, false><<<c.count, kBlock, 0, s>>>(a, c.tile0, c.base, 0, k)));
            }
        } else if (listed) {
            PDLPX_SHAPE_SWITCH(c.shape, (packDual<GG, RR, UU, true><<<c.count, kBlock, 0, s>>>(a, c.tile0, c.base, c.list0, k)));
        } else {
            PDLPX_SHAPE_SWITCH(c.shape, (packDual<GG, RR, UU, false><<<c.count, kBlock, 0, s>>>(a, c.tile0, c.base, 0, k)));
        }
    }

    int launchCycle(int N, bool steps = true) {
        int n = 0;
        const PackArgs& a = args;
        for (int k = 1; k <= (steps ? N : 0); ++k) {
            for (const Launch& c : lc) {
                launchPrimal(c, k);
                ++n;
            }
            for (const Launch& c : lr) {
                launchDual(c, k);
                ++n;
            }
        }
        for (const Launch& c : lr) {
            if (listed) {
                PDLPX_G_SWITCH(checkGroup(c.shape), (packCheckRows<GG, true><<<c.count, kBlock, 0, s>>>(a, c.tile0, c.list0)));
            } else {
                PDLPX_G_SWITCH(checkGroup(c.shape), (packCheckRows<GG, false><<<c.count, kBlock, 0, s>>>(a, c.tile0, 0)));
            }
            ++n;
        }
        for (const Launch& c : lc) {
            if (listed) {
                PDLPX_G_SWITCH(checkGroup(c.shape), (packCheckCols<GG, true><<<c.count, kBlock, 0, s>>>(a, c.tile0, c.list0)));
            } else {
                PDLPX_G_SWITCH(checkGroup(c.shape), (packCheckCols<GG, false><<<c.count, kBlock, 0, s>>>(a, c.tile0, 0)));
            }
            ++n;
        }
        packController<<<(L + kCtlWarps - 1) / kCtlWarps, 32 * kCtlWarps, 0, s>>>(a);
        if (live_ct + live_rt > 0) packRestart<<<live_ct + live_rt, kBlock, 0, s>>>(a, live_ct, listed ? 1 : 0);
        packFinish<<<(L + 127) / 128, 128, 0, s>>>(a);
        packModes<<<(nct + nrt + 255) / 256, 256, 0, s>>>(a);
        return n + 4;
    }

    int launchPower(int chunk) {
        int n = 0;
        const PackArgs& a = args;
        for (int it = 0; it < chunk; ++it) {
            for (const Launch& c : cls_r) {
                PDLPX_G_SWITCH(checkGroup(c.shape), (packPowerA<GG><<<c.count, kBlock, 0, s>>>(a, c.tile0)));
                ++n;
            }
            for (const Launch& c : cls_c) {
                PDLPX_G_SWITCH(checkGroup(c.shape), (packPowerAt<GG><<<c.count, kBlock, 0, s>>>(a, c.tile0)));
                ++n;
            }
            packPowerFinish1<<<(L + kCtlWarps - 1) / kCtlWarps, 32 * kCtlWarps, 0, s>>>(a);
            packPowerNormalize<<<nct, kBlock, 0, s>>>(a);
            packPowerFinish2<<<(L + kCtlWarps - 1) / kCtlWarps, 32 * kCtlWarps, 0, s>>>(a);
            n += 3;
        }
        return n;
    }
};

// Controller constants and initial solver state of one LP (as the single-LP
// solve sets them up); nb_rows / nb_cols are its partial counts.
void lpState(const Item& it, const pdlpx_options& o, bool mixed, int nb_rows, int nb_cols, DevConst& dc, DevState& st) {
    const ScaledLp& sc = it.sc;
    const int32_t m = it.lp.m, n = it.lp.n;
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
    dc.nb_rows = nb_rows;
    dc.nb_cols = nb_cols;
    dc.stall_limit = 10;
    dc.ref_fixed = o.reference_fixed_columns != 0;
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
    dc.noise_factor = 1.0;
    st.step = 1.0;
    st.pw = o.primal_weight;
    st.prec = mixed ? 0 : 1;
    st.fpe0 = -1.0;
    st.last_fpe = std::numeric_limits<double>::infinity();
    st.best_pw = st.pw;
    st.best_score = std::numeric_limits<double>::infinity();
    st.best_kkt = std::numeric_limits<double>::infinity();
    st.precond_pw = sc.precond_pw;
    st.switch_total = -1;
}

// Host image of one LP's share of the pack, in the pack numbering (renumbered
// sides, padded rows and columns included).
void stageItem(const Pack& pk, const Item& it, const pdlpx_options& o, char* img, char* iters) {
    const ScaledLp& sc = it.sc;
    const int32_t m = it.lp.m, n = it.lp.n;
    const int64_t r0 = it.r0, c0 = it.c0, za = it.za, zt = it.zt, mp = it.mp, np = it.np;
    const SideOrder& co = it.cols;
    const SideOrder& ro = it.rows;
    const double inf = std::numeric_limits<double>::infinity();
    auto I = [&](size_t off) { return reinterpret_cast<int32_t*>(img + off); };
    auto F = [&](size_t off) { return reinterpret_cast<float*>(img + off); };
    auto D = [&](size_t off) { return reinterpret_cast<double*>(img + off); };
    // CSR of A (rows in pack order, columns renumbered) and of A^T; an entry keeps
    // its place inside its row
    {
        int32_t* ptr = I(pk.o_aptr) + r0;
        int32_t* idx = I(pk.o_aidx) + za;
        double* v64 = D(pk.o_av64) + za;
        float* v32 = pk.mixed ? F(pk.o_av32) + za : nullptr;
        int64_t k = 0;
        for (int64_t i = 0; i < mp; ++i) {
            ptr[i] = static_cast<int32_t>(za + k);
            if (i >= m) continue;
            const int32_t old = ro.order[i];
            for (int32_t q = sc.a.ptr[old]; q < sc.a.ptr[old + 1]; ++q, ++k) {
                idx[k] = static_cast<int32_t>(c0 + co.pos[sc.a.idx[q]]);
                v64[k] = sc.a.val[q];
                if (v32) v32[k] = static_cast<float>(sc.a.val[q]);
            }
        }
    }
    {
        int32_t* ptr = I(pk.o_atptr) + c0;
        int32_t* idx = I(pk.o_atidx) + zt;
        double* v64 = D(pk.o_atv64) + zt;
        float* v32 = pk.mixed ? F(pk.o_atv32) + zt : nullptr;
        int64_t k = 0;
        for (int64_t j = 0; j < np; ++j) {
            ptr[j] = static_cast<int32_t>(zt + k);
            if (j >= n) continue;
            const int32_t old = co.order[j];
            for (int32_t q = sc.at.ptr[old]; q < sc.at.ptr[old + 1]; ++q, ++k) {
                idx[k] = static_cast<int32_t>(r0 + ro.pos[sc.at.idx[q]]);
                v64[k] = sc.at.val[q];
                if (v32) v32[k] = static_cast<float>(sc.at.val[q]);
            }
        }
    }
    // sliced ELL of the renumbered sides that use it: slice s of the LP holds its
    // rows 32 s .. 32 s + 31, entry k of lane l at first + k * 32 + l
    auto sell = [&](const SideOrder& so, const Csr& a, const SideOrder& other, int64_t row0, int64_t other0,
                    int64_t e0, size_t o_hdr, size_t o_idx, size_t o_v32, size_t o_v64) {
        int2* hdr = reinterpret_cast<int2*>(img + o_hdr) + row0 / kSlice;
        int32_t* idx = I(o_idx);
        double* v64 = D(o_v64);
        float* v32 = pk.mixed ? F(o_v32) : nullptr;
        int64_t e = e0;
        const int32_t rows = static_cast<int32_t>(so.order.size());
        for (size_t s = 0; s < so.slice_len.size(); ++s) {
            const int32_t len = so.slice_len[s];
            hdr[s] = make_int2(static_cast<int>(e), len);
            for (int32_t lane = 0; lane < kSlice; ++lane) {
                const int64_t r = static_cast<int64_t>(s) * kSlice + lane;
                const int32_t old = r < rows ? so.order[r] : -1;
                const int32_t b = old >= 0 ? a.ptr[old] : 0, cnt = old >= 0 ? a.ptr[old + 1] - b : 0;
                for (int32_t k = 0; k < len; ++k) {
                    const int64_t at = e + static_cast<int64_t>(k) * kSlice + lane;
                    const bool real = k < cnt;
                    idx[at] = static_cast<int32_t>(real ? other0 + other.pos[a.idx[b + k]] : other0);
                    v64[at] = real ? a.val[b + k] : 0.0;
                    if (v32) v32[at] = real ? static_cast<float>(a.val[b + k]) : 0.0f;
                }
            }
            e += static_cast<int64_t>(len) * kSlice;
        }
    };
    if (isSell(it.shapeP)) sell(co, sc.at, ro, c0, r0, it.ec, pk.o_chdr, pk.o_cidx, pk.o_cv32, pk.o_cv64);
    if (isSell(it.shapeD)) sell(ro, sc.a, co, r0, c0, it.er, pk.o_rhdr, pk.o_ridx, pk.o_rv32, pk.o_rv64);
    // per-column / per-row constants; padding is empty, free, zero cost, unit scales
    for (int64_t j = 0; j < np; ++j) {
        const bool real = j < n;
        const int32_t old = real ? co.order[j] : 0;
        const double c = real ? sc.c[old] : 0.0, lb = real ? sc.cl[old] : -inf, ub = real ? sc.cu[old] : inf;
        const double tau = real ? sc.tau[old] : 1.0, cs = real ? sc.col_scale[old] : 1.0;
        reinterpret_cast<ColPack<double>*>(img + pk.o_cp64)[c0 + j] = ColPack<double>{c, lb, ub, tau};
        if (pk.mixed)
            reinterpret_cast<ColPack<float>*>(img + pk.o_cp32)[c0 + j] =
                ColPack<float>{static_cast<float>(c), static_cast<float>(lb), static_cast<float>(ub), static_cast<float>(tau)};
        D(pk.o_c)[c0 + j] = c;
        D(pk.o_lb)[c0 + j] = lb;
        D(pk.o_ub)[c0 + j] = ub;
        D(pk.o_cs)[c0 + j] = cs;
        D(pk.o_tau)[c0 + j] = tau;
    }
    for (int64_t i = 0; i < mp; ++i) {
        const bool real = i < m;
        const int32_t old = real ? ro.order[i] : 0;
        const double sig = real ? sc.sigma[old] : 1.0, rl = real ? sc.rl[old] : -inf, ru = real ? sc.ru[old] : inf;
        const double type = real ? static_cast<double>(sc.row_type[old]) : static_cast<double>(kRowRanged);
        const double rs = real ? sc.row_scale[old] : 1.0;
        reinterpret_cast<RowPack<double>*>(img + pk.o_rp64)[r0 + i] = RowPack<double>{sig, rl, ru, type};
        if (pk.mixed)
            reinterpret_cast<RowPack<float>*>(img + pk.o_rp32)[r0 + i] =
                RowPack<float>{static_cast<float>(sig), static_cast<float>(rl), static_cast<float>(ru), static_cast<float>(type)};
        D(pk.o_rl)[r0 + i] = rl;
        D(pk.o_ru)[r0 + i] = ru;
        D(pk.o_rs)[r0 + i] = rs;
        D(pk.o_sig)[r0 + i] = sig;
    }
    // tiles: (LP, mode, first, end) -- padded tiles are whole
    const int initial_mode = pk.mixed ? kModeFp32 : kModeFp64;
    const int tp = tileRows(it.shapeP), td = tileRows(it.shapeD);
    for (int k = 0; k < it.nct; ++k)
        reinterpret_cast<int4*>(img + pk.o_ctinfo)[it.ct0 + k] =
            make_int4(it.l, initial_mode, static_cast<int>(c0 + int64_t(k) * tp), static_cast<int>(c0 + int64_t(k + 1) * tp));
    for (int k = 0; k < it.nrt; ++k)
        reinterpret_cast<int4*>(img + pk.o_rtinfo)[it.rt0 + k] =
            make_int4(it.l, initial_mode, static_cast<int>(r0 + int64_t(k) * td), static_cast<int>(r0 + int64_t(k + 1) * td));
    reinterpret_cast<int4*>(img + pk.o_lpt)[it.l] = make_int4(it.ct0, it.nct, it.rt0, it.nrt);
    // power-iteration start vector: mt19937(42) normals over the original columns,
    // normalised (pdlp.cpp:1990-2001), placed in the pack numbering; zero on padding
    {
        double* x0 = D(pk.o_pix) + c0;
        std::vector<double> g(n);
        std::mt19937 rng(42);
        std::normal_distribution<double> dist(0.0, 1.0);
        double xn = 0.0;
        for (int32_t j = 0; j < n; ++j) {
            g[j] = dist(rng);
            xn += g[j] * g[j];
        }
        xn = std::sqrt(xn);
        if (xn < 1e-15) xn = 1.0;
        for (int32_t j = 0; j < n; ++j) x0[co.pos[j]] = g[j] / xn;
        for (int64_t j = n; j < np; ++j) x0[j] = 0.0;
    }
    // controller constants and initial state (as the single-LP solve)
    DevConst dc{};
    DevState st{};
    lpState(it, o, pk.mixed, it.nrt, it.nct, dc, st);
    reinterpret_cast<DevConst*>(img + pk.o_dc)[it.l] = dc;
    reinterpret_cast<DevState*>(img + pk.o_st)[it.l] = st;
    reinterpret_cast<PowerState*>(img + pk.o_ps)[it.l] = PowerState{1.0, 0.0, 0.0, 0, o.sv_max_iter <= 0 ? 1 : 0};
    // warm start, scaled like pdlp.cpp:1812-1827 (iters is null when no LP of the pack has one)
    if (iters == nullptr) return;
    // iterate arrays start at image_end in the arena and at 0 in `iters`
    auto IF = [&](size_t off) { return reinterpret_cast<float*>(iters + (off - pk.image_end)); };
    auto ID = [&](size_t off) { return reinterpret_cast<double*>(iters + (off - pk.image_end)); };
    const bool warm = !it.warm_x.empty();
    std::vector<double> wx(n, 0.0), wy(m, 0.0);  // pack numbering
    if (warm) {
        for (int32_t j = 0; j < n; ++j) wx[co.pos[j]] = it.warm_x[j] / sc.col_scale[j] * sc.con_scale;
        for (int32_t i = 0; i < m; ++i)
            wy[ro.pos[i]] = it.warm_y[i] * sc.obj_scale / (sc.obj_sign * sc.row_scale[i]);
    }
    if (pk.mixed) {
        for (int32_t j = 0; j < n; ++j) {
            const float f = static_cast<float>(wx[j]);
            IF(pk.o_xi32)[c0 + j] = f;
            IF(pk.o_xr32)[c0 + j] = f;
            IF(pk.o_xh32)[c0 + j] = f;
            ID(pk.o_xc)[c0 + j] = f;
        }
        for (int32_t i = 0; i < m; ++i) {
            const float f = static_cast<float>(wy[i]);
            IF(pk.o_yi32)[r0 + i] = f;
            IF(pk.o_yh32)[r0 + i] = f;
            ID(pk.o_yc)[r0 + i] = f;
        }
    } else {
        const size_t xs[4] = {pk.o_xc, pk.o_xi64, pk.o_xr64, pk.o_xh64};
        const size_t ys[3] = {pk.o_yc, pk.o_yi64, pk.o_yh64};
        for (size_t off : xs) std::memcpy(ID(off) + c0, wx.data(), 8 * static_cast<size_t>(n));
        for (size_t off : ys) std::memcpy(ID(off) + r0, wy.data(), 8 * static_cast<size_t>(m));
    }
}

bool timeUp(std::chrono::steady_clock::time_point t0, double lim) {
    if (lim < 0.0) return false;
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >= lim;
}

// Status, unscaled solution and result record of one LP from its final solver
// state and its pdhg iterates xs, ys (scaled space, original numbering).
void finishOutcome(const Item& it, const DevState& f, const std::vector<double>& xs, const std::vector<double>& ys,
                   bool mixed, bool out_of_time, double secs, double dev_s, int launches, LpOutcome& out) {
    const int32_t m = it.lp.m, n = it.lp.n;
    int32_t status;
    if (f.done) {
        status = f.status;
        if (status == PDLPX_STATUS_ITER_LIMIT && out_of_time) status = PDLPX_STATUS_TIME_LIMIT;
    } else {
        status = f.converged ? PDLPX_STATUS_OPTIMAL : PDLPX_STATUS_TIME_LIMIT;
    }
    const ScaledLp& sc = it.sc;
    out.x.assign(n, 0.0);
    out.y.assign(m, 0.0);
    double obj = 0.0;
    if (status == PDLPX_STATUS_OPTIMAL) {
        const double ic = 1.0 / sc.con_scale, io = 1.0 / sc.obj_scale;
        double ov = it.lp.offset;
        for (int32_t j = 0; j < n; ++j) {
            double xj = xs[j] * sc.col_scale[j] * ic;
            if (std::isfinite(it.lp.cl[j])) xj = std::max(xj, it.lp.cl[j]);
            if (std::isfinite(it.lp.cu[j])) xj = std::min(xj, it.lp.cu[j]);
            out.x[j] = xj;
            ov += it.lp.obj[j] * xj;
        }
        for (int32_t i = 0; i < m; ++i) out.y[i] = sc.obj_sign * ys[i] * sc.row_scale[i] * io;
        obj = ov;
    } else if (status == PDLPX_STATUS_INFEASIBLE) {
        const double io = 1.0 / sc.obj_scale;
        for (int32_t i = 0; i < m; ++i) out.y[i] = sc.obj_sign * ys[i] * sc.row_scale[i] * io;
    } else if (status == PDLPX_STATUS_UNBOUNDED) {
        const double ic = 1.0 / sc.con_scale;
        for (int32_t j = 0; j < n; ++j) out.x[j] = xs[j] * sc.col_scale[j] * ic;
    }
    pdlpx_result& r = out.r;
    std::memset(&r, 0, sizeof(r));
    r.status = status;
    r.objective = obj;
    r.iterations = f.total;
    r.work_units = static_cast<double>(f.total) * (4.0 * static_cast<double>(sc.a.nnz()) + 2.0 * static_cast<double>(m + n));
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
    r.device_seconds = dev_s;
    r.used_gpu = 1;
    r.kernel_launches = launches;
}

// Read one finished (or stopped) LP back from the device and unscale it
// (pdlp.cpp:2678-2712): x = x_hat * col_scale / con_scale clamped to the
// original bounds, y = sign * y_hat * row_scale / obj_scale, in the LP's
// original numbering.
int32_t collectLp(const Pack& pk, int l, bool out_of_time, double secs, double dev_s, int launches, LpOutcome& out,
                  std::string& err) {
    const Item& it = *pk.items[l];
    cudaStream_t s = pk.s;
    const int32_t m = it.lp.m, n = it.lp.n;
    DevState f{};
    PDLPX_BCK(cudaMemcpyAsync(&f, pk.args.st + l, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    PDLPX_BCK(cudaStreamSynchronize(s));
    std::vector<double> xs(n), ys(m);  // original numbering, scaled space
    if (f.prec == 0) {
        std::vector<float> fx(it.np), fy(it.mp);
        PDLPX_BCK(cudaMemcpyAsync(fx.data(), pk.args.it32.xh + it.c0, 4 * fx.size(), cudaMemcpyDeviceToHost, s));
        PDLPX_BCK(cudaMemcpyAsync(fy.data(), pk.args.it32.yh + it.r0, 4 * fy.size(), cudaMemcpyDeviceToHost, s));
        PDLPX_BCK(cudaStreamSynchronize(s));
        for (int32_t j = 0; j < n; ++j) xs[j] = fx[it.cols.pos[j]];
        for (int32_t i = 0; i < m; ++i) ys[i] = fy[it.rows.pos[i]];
    } else {
        std::vector<double> dx(it.np), dy(it.mp);
        PDLPX_BCK(cudaMemcpyAsync(dx.data(), pk.args.it64.xh + it.c0, 8 * dx.size(), cudaMemcpyDeviceToHost, s));
        PDLPX_BCK(cudaMemcpyAsync(dy.data(), pk.args.it64.yh + it.r0, 8 * dy.size(), cudaMemcpyDeviceToHost, s));
        PDLPX_BCK(cudaStreamSynchronize(s));
        for (int32_t j = 0; j < n; ++j) xs[j] = dx[it.cols.pos[j]];
        for (int32_t i = 0; i < m; ++i) ys[i] = dy[it.rows.pos[i]];
    }
    finishOutcome(it, f, xs, ys, pk.mixed, out_of_time, secs, dev_s, launches, out);
    return PDLPX_OK;
}

// Build and run one pack; `done(l, outcome)` is called from this thread for
// every LP as soon as a cycle finds it finished (and for the rest when the
// time limit or `stop` ends the pack).
int32_t solvePack(Pack& pk, const pdlpx_options& o, std::chrono::steady_clock::time_point t0,
                  const std::atomic<int>* stop, const LpDone& done, std::string& err) {
    const int L = pk.L;
    for (int l = 0; l < L; ++l) pk.items[l]->l = l;
    pk.place();
    pk.layout();
    bool any_warm = false;
    for (const Item* it : pk.items) any_warm |= !it->warm_x.empty();

    // host image: everything the kernels read, filled per LP in parallel
    std::unique_ptr<char[]> img(new char[pk.image_end]);
    std::unique_ptr<char[]> iters(any_warm ? new char[pk.iter_end - pk.image_end] : nullptr);
    if (any_warm) std::memset(iters.get(), 0, pk.iter_end - pk.image_end);
    reinterpret_cast<int32_t*>(img.get() + pk.o_aptr)[pk.M] = static_cast<int32_t>(pk.Z);
    reinterpret_cast<int32_t*>(img.get() + pk.o_atptr)[pk.Nc] = static_cast<int32_t>(pk.Z);
    parallelFor(L, [&](int l) { stageItem(pk, *pk.items[l], o, img.get(), iters.get()); });

    PDLPX_BCK(cudaStreamCreateWithFlags(&pk.s, cudaStreamNonBlocking));
    PDLPX_BCK(cudaMallocAsync(reinterpret_cast<void**>(&pk.d), pk.total, pk.s));
    cudaStream_t s = pk.s;
    PDLPX_BCK(cudaMemcpyAsync(pk.d, img.get(), pk.image_end, cudaMemcpyHostToDevice, s));
    if (any_warm)
        PDLPX_BCK(cudaMemcpyAsync(pk.d + pk.image_end, iters.get(), pk.iter_end - pk.image_end, cudaMemcpyHostToDevice, s));
    else
        PDLPX_BCK(cudaMemsetAsync(pk.d + pk.image_end, 0, pk.iter_end - pk.image_end, s));
    PDLPX_BCK(cudaMemsetAsync(pk.d + pk.iter_end, 0, pk.total - pk.iter_end, s));
    pk.makeArgs(o);

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    PDLPX_BCK(cudaEventCreate(&ev0));
    PDLPX_BCK(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } ev_guard{ev0, ev1};
    PDLPX_BCK(cudaEventRecord(ev0, s));
    int launches = 0;
    auto deviceSeconds = [&]() -> double {
        float ms = 0.0f;
        if (cudaEventRecord(ev1, s) == cudaSuccess && cudaEventSynchronize(ev1) == cudaSuccess)
            cudaEventElapsedTime(&ms, ev0, ev1);
        return 1e-3 * ms;
    };
    auto hostSeconds = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };

    // counters[0] / per-LP flags (pageable: a pinned allocation would
    // synchronize the device, which other packs share)
    std::vector<int> h_flags(std::max(L, 16));
    int* h_small = h_flags.data();

    auto capture = [&](cudaGraphExec_t& g, int& count, bool power) -> int32_t {
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
        cudaGraph_t graph = nullptr;
        PDLPX_BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        count = power ? pk.launchPower(8) : pk.launchCycle(o.termination_eval_frequency, !pk.persist);
        PDLPX_BCK(cudaStreamEndCapture(s, &graph));
        const cudaError_t ie = cudaGraphInstantiate(&g, graph, 0);
        cudaGraphDestroy(graph);
        PDLPX_BCK(ie);
        return PDLPX_OK;
    };
    auto stopped = [&]() { return stop != nullptr && stop->load(std::memory_order_relaxed) != 0; };

    // ---- power iteration of every LP
    if (o.sv_max_iter > 0) {
        int32_t rc = capture(pk.power, pk.power_launches, true);
        if (rc != PDLPX_OK) return rc;
        for (int guard = 0; guard < 2 + o.sv_max_iter / 8; ++guard) {
            PDLPX_BCK(cudaGraphLaunch(pk.power, s));
            launches += pk.power_launches;
            PDLPX_BCK(cudaMemcpyAsync(h_small, pk.args.counters, 4, cudaMemcpyDeviceToHost, s));
            PDLPX_BCK(cudaStreamSynchronize(s));
            if (h_small[0] >= L || stopped()) break;
        }
    }
    packInitStep<<<(L + 127) / 128, 128, 0, s>>>(pk.args);
    ++launches;
    PDLPX_BCK(cudaGetLastError());

    // ---- autotuner (option autotune): per sliced-ELL class and side, time
    // three launches of each entries-per-round variant on the pack itself and
    // keep the fastest (a variant must beat the table's pick by 3%).  The
    // variants give identical results, so the choice never changes an LP's
    // solution; the timing launches' writes to the iterates are undone by
    // re-uploading the initial iterates.
    if (o.autotune) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        PDLPX_BCK(cudaEventCreate(&e0));
        PDLPX_BCK(cudaEventCreate(&e1));
        struct EvPair {
            cudaEvent_t a, b;
            ~EvPair() {
                cudaEventDestroy(a);
                cudaEventDestroy(b);
            }
        } evp{e0, e1};
        for (int side = 0; side < 2; ++side)
            for (Launch& c : side == 0 ? pk.cls_c : pk.cls_r) {
                if (!isSell(c.shape) || c.count == 0) continue;
                float best = 0.0f;
                int pick = c.shape;
                for (int cand : {c.shape, kNumShapes + 0, kNumShapes + 1, kNumShapes + 2}) {
                    if (cand == c.shape && best > 0.0f) continue;
                    c.kern = cand;
                    for (int r = 0; r < 4; ++r) {  // one warm-up, three timed
                        if (r == 1) PDLPX_BCK(cudaEventRecord(e0, s));
                        side == 0 ? pk.launchPrimal(c, 1) : pk.launchDual(c, 1);
                    }
                    PDLPX_BCK(cudaEventRecord(e1, s));
                    PDLPX_BCK(cudaGetLastError());
                    PDLPX_BCK(cudaEventSynchronize(e1));
                    float ms = 0.0f;
                    PDLPX_BCK(cudaEventElapsedTime(&ms, e0, e1));
                    launches += 4;
                    if (best == 0.0f || ms < 0.97f * best) {
                        best = ms;
                        pick = cand;
                    }
                }
                c.kern = pick;
            }
        pk.lc = pk.cls_c;
        pk.lr = pk.cls_r;
        if (any_warm)
            PDLPX_BCK(cudaMemcpyAsync(pk.d + pk.image_end, iters.get(), pk.iter_end - pk.image_end,
                                      cudaMemcpyHostToDevice, s));
        else
            PDLPX_BCK(cudaMemsetAsync(pk.d + pk.image_end, 0, pk.iter_end - pk.image_end, s));
        if (o.verbose) {
            for (int side = 0; side < 2; ++side)
                for (const Launch& c : side == 0 ? pk.cls_c : pk.cls_r)
                    if (isSell(c.shape) && c.count > 0)
                        std::printf("PDLP batch autotune: %s sliced-ELL class U%d -> U%d (%d tiles)\n",
                                    side == 0 ? "primal" : "dual", kSellU[c.shape - kNumShapes],
                                    kSellU[c.k() - kNumShapes], c.count);
            std::fflush(stdout);
        }
    }

    // ---- persistent cycle (option batch_persistent): the steps of a cycle as
    // one cooperative launch ahead of the graph of its check, controller and
    // restart launches
    if (o.batch_persistent && pk.persistable()) {
        int nb = 0, dev = 0, sms = 0, coop = 0;
        PDLPX_BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, packCycleSell, kBlock, 0));
        PDLPX_BCK(cudaGetDevice(&dev));
        PDLPX_BCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        PDLPX_BCK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        if (nb > 0 && coop) {
            pk.persist_grid = std::max(1, std::min(nb * sms, std::max(pk.nct, pk.nrt)));
            PDLPX_BCK(cudaMallocAsync(reinterpret_cast<void**>(&pk.pd),
                                      16 + sizeof(int4) * static_cast<size_t>(pk.nct + pk.nrt), s));
            pk.persist = true;
            PDLPX_BCK(pk.uploadPersistTiles());
        }
    }

    // ---- restart cycles; finished LPs are read back after the cycle that ends them
    {
        int32_t rc = capture(pk.cycle, pk.cycle_launches, false);
        if (rc != PDLPX_OK) return rc;
    }
    int perr = 0;
    SleepWait sleeper;
    std::vector<char> keep(L, 1), collected(L, 0);
    std::vector<int> cl, rl;
    int cycles = 0, ncollected = 0;
    while (ncollected < L) {
        if (timeUp(t0, o.max_solve_seconds) || stopped()) break;
        if (pk.persist) {
            PDLPX_BCK(pk.launchPersistent(o.termination_eval_frequency));
            ++launches;
        }
        PDLPX_BCK(cudaGraphLaunch(pk.cycle, s));
        launches += pk.cycle_launches;
        ++cycles;
        PDLPX_BCK(sleeper.wait(s));
        PDLPX_BCK(cudaMemcpyAsync(h_small, pk.args.flags, 4 * static_cast<size_t>(L), cudaMemcpyDeviceToHost, s));
        if (pk.persist) PDLPX_BCK(cudaMemcpyAsync(&perr, pk.pd + 8, 4, cudaMemcpyDeviceToHost, s));
        PDLPX_BCK(cudaStreamSynchronize(s));
        if (perr != 0) {
            err = "persistent cycle: a grid barrier ran out of polls";
            return PDLPX_E_TIMEOUT;
        }
        int done_count = 0, fp64 = 0, live_tiles = 0;
        bool fresh = false;
        for (int l = 0; l < L; ++l) {
            done_count += h_small[l] & 1;
            fp64 += (h_small[l] >> 1) & 1;
            if (!(h_small[l] & 1)) live_tiles += pk.items[l]->nct + pk.items[l]->nrt;
            fresh |= (h_small[l] & 1) && !collected[l];
        }
        if (fresh) {
            const double dev_s = deviceSeconds(), secs = hostSeconds();
            for (int l = 0; l < L; ++l) {
                if (!(h_small[l] & 1) || collected[l]) continue;
                LpOutcome out;
                const int32_t rc = collectLp(pk, l, false, secs, dev_s, launches, out, err);
                if (rc != PDLPX_OK) return rc;
                collected[l] = 1;
                ++ncollected;
                done(l, std::move(out));
            }
        }
        if (o.verbose && cycles % 10 == 0) {
            std::printf("PDLP batch  %7d iterations per LP  %d/%d LPs done  %d on FP64 iterates  %d live tiles  %.3fs  [B200]\n",
                        cycles * o.termination_eval_frequency, done_count, L, fp64, live_tiles, hostSeconds());
            std::fflush(stdout);
        }
        if (done_count >= L) break;
        if (o.batch_compact && live_tiles < ((pk.live_ct + pk.live_rt) * 3) / 5) {
            for (int l = 0; l < L; ++l) keep[l] = !(h_small[l] & 1);
            pk.liveLists(keep, cl, rl);
            if (!cl.empty())
                PDLPX_BCK(cudaMemcpyAsync(pk.d + pk.o_clist, cl.data(), 4 * cl.size(), cudaMemcpyHostToDevice, s));
            if (!rl.empty())
                PDLPX_BCK(cudaMemcpyAsync(pk.d + pk.o_rlist, rl.data(), 4 * rl.size(), cudaMemcpyHostToDevice, s));
            if (pk.persist) PDLPX_BCK(pk.uploadPersistTiles());
            int32_t rc = capture(pk.cycle, pk.cycle_launches, false);
            if (rc != PDLPX_OK) return rc;
        }
    }
    // LPs the time limit or the stop request left unfinished
    if (ncollected < L) {
        const double dev_s = deviceSeconds(), secs = hostSeconds();
        const bool out_of_time = timeUp(t0, o.max_solve_seconds);
        for (int l = 0; l < L; ++l) {
            if (collected[l]) continue;
            LpOutcome out;
            const int32_t rc = collectLp(pk, l, out_of_time, secs, dev_s, launches, out, err);
            if (rc != PDLPX_OK) return rc;
            done(l, std::move(out));
        }
    }
    return PDLPX_OK;
}

// Launch shape of one matrix side in the batch: a pinned shape (1..16 CSR,
// 17..19 sliced ELL with 4 / 8 / 16 entries per round), a forced lane count,
// sliced ELL for mean row lengths up to 32, else the batch CSR table.
int batchSideShape(int pinned, int group, bool sell, int64_t nnz, int32_t rows) {
    if (pinned > kNumShapes && pinned <= kNumShapes + kNumSell) return pinned - 1;
    if (pinned > 0 || group > 0) return chooseShape(pinned, group, nnz, rows, true);
    const double mean = rows > 0 ? static_cast<double>(nnz) / rows : 0.0;
    // measured on 512 lognormal-sized LPs (mean 8 / 20 entries per column / row,
    // us per iteration of the full pack, FP32 / FP64 phase): 4 entries per round
    // on the columns and 8 on the rows 127 / 132; 8 and 8: 181 / 171
    if (sell && mean <= 32.0) return kNumShapes + (mean <= 12.0 ? 0 : 1);
    return batchShape(nnz, rows);
}

// Copy, validate and scale one LP; choose its launch shapes and storage.
int32_t prepareItem(const pdlpx_lp& in, const pdlpx_options& o, Item& it) {
    HostLp& lp = it.lp;
    lp.m = in.m;
    lp.n = in.n;
    lp.maximize = in.sense == PDLPX_MAXIMIZE;
    if (in.m < 0 || in.n < 0 || !canonicalCsr(in.m, in.n, in.nnz, in.row_ptr, in.col_idx, in.val, lp.a) ||
        (in.n > 0 && (in.obj == nullptr || in.col_lb == nullptr || in.col_ub == nullptr)) ||
        (in.m > 0 && (in.row_lb == nullptr || in.row_ub == nullptr)))
        return PDLPX_E_INVALID;
    lp.obj.assign(in.obj, in.obj + in.n);
    lp.cl.assign(in.col_lb, in.col_lb + in.n);
    lp.cu.assign(in.col_ub, in.col_ub + in.n);
    lp.rl.assign(in.row_lb, in.row_lb + in.m);
    lp.ru.assign(in.row_ub, in.row_ub + in.m);
    lp.offset = in.obj_offset;
    if (in.warm_x != nullptr && in.warm_y != nullptr) {
        it.warm_x.assign(in.warm_x, in.warm_x + in.n);
        it.warm_y.assign(in.warm_y, in.warm_y + in.m);
    }
    it.trivial = lp.m == 0 || lp.n == 0;
    if (it.trivial) return PDLPX_OK;
    const bool mixed = o.precision != PDLPX_PREC_FP64;
    buildScaled(lp, o, it.sc, ruizFor(o, lp.a.nnz(), &it.scale_note));
    const int64_t z = it.sc.a.nnz();
    it.shapeP = batchSideShape(o.shape_primal, o.spmv_group_at, o.batch_sell != 0, z, lp.n);
    it.shapeD = batchSideShape(o.shape_dual, o.spmv_group_a, o.batch_sell != 0, z, lp.m);
    const int tp = tileRows(it.shapeP), td = tileRows(it.shapeD);
    it.nct = static_cast<int>((static_cast<int64_t>(lp.n) + tp - 1) / tp);
    it.nrt = static_cast<int>((static_cast<int64_t>(lp.m) + td - 1) / td);
    it.np = static_cast<int64_t>(it.nct) * tp;
    it.mp = static_cast<int64_t>(it.nrt) * td;
    orderSide(it.sc.at.ptr, lp.n, it.np, isSell(it.shapeP), it.cols);
    orderSide(it.sc.a.ptr, lp.m, it.mp, isSell(it.shapeD), it.rows);
    it.bytes = itemBytes(it, mixed);
    return PDLPX_OK;
}

// Closed-form LPs (no rows or no columns) through the single-LP engine's host
// path (pdlp.cpp:812-860).
int32_t solveTrivialItem(const Item& it, const pdlpx_options& o, LpOutcome& out, std::string& err) {
    Engine e;
    e.setOptions(o);
    const HostLp& lp = it.lp;
    int32_t rc = e.load(lp.m, lp.n, lp.a.nnz(), lp.a.ptr.data(), lp.a.idx.data(), lp.a.val.data(), lp.obj.data(),
                        lp.cl.data(), lp.cu.data(), lp.rl.data(), lp.ru.data(),
                        lp.maximize ? PDLPX_MAXIMIZE : PDLPX_MINIMIZE, lp.offset);
    if (rc == PDLPX_OK) rc = e.solve(&out.r);
    if (rc != PDLPX_OK) {
        err = e.last_error;
        return rc;
    }
    out.x = e.primal();
    out.y = e.dual();
    return PDLPX_OK;
}

bool optionsSupported(const pdlpx_options& o, std::string& err) {
    if (o.anderson_acceleration && o.anderson_window_size >= 2) {
        err = "anderson_acceleration is not available in the device engine";
        return false;
    }
    if (o.adaptive_step) {
        err = "adaptive_step is not available in the batched solve";
        return false;
    }
    if (o.termination_eval_frequency <= 0) {
        err = "termination_eval_frequency must be positive";
        return false;
    }
    return true;
}

int32_t selectDevice(const pdlpx_options& o, std::string& err) {
    int devcount = 0;
    if (cudaGetDeviceCount(&devcount) != cudaSuccess || devcount <= 0) {
        err = "no CUDA device visible";
        return PDLPX_E_NO_DEVICE;
    }
    PDLPX_BCK(cudaSetDevice((o.device >= 0 && o.device < devcount) ? o.device : 0));
    return PDLPX_OK;
}

// Solve one pack of prepared items on the current device.
int32_t runPack(const std::vector<Item*>& items, const pdlpx_options& o, std::chrono::steady_clock::time_point t0,
                const std::atomic<int>* stop, const LpDone& done, std::string& err) {
    Pack pk;
    pk.mixed = o.precision != PDLPX_PREC_FP64;
    pk.items = items;
    pk.L = static_cast<int>(items.size());
    if (pk.L == 0) return PDLPX_OK;
    return solvePack(pk, o, t0, stop, done, err);
}

#include "family.cuh"

}  // namespace

struct PreparedLp {
    Item item;
};

void PreparedLpDeleter::operator()(PreparedLp* p) const { delete p; }

int32_t prepareLp(const pdlpx_lp& lp, const pdlpx_options& o, PreparedPtr& out, std::string& err) {
    if (!optionsSupported(o, err)) return PDLPX_E_INVALID;
    PreparedPtr p(new PreparedLp());
    const int32_t rc = prepareItem(lp, o, p->item);
    if (rc != PDLPX_OK) {
        err = "invalid LP (CSR structure, sizes or missing arrays)";
        return rc;
    }
    out = std::move(p);
    return PDLPX_OK;
}

bool preparedTrivial(const PreparedLp& p) { return p.item.trivial; }
size_t preparedBytes(const PreparedLp& p) { return p.item.bytes; }
int32_t preparedRows(const PreparedLp& p) { return p.item.lp.m; }
int32_t preparedCols(const PreparedLp& p) { return p.item.lp.n; }

int32_t solvePreparedTrivial(const PreparedLp& p, const pdlpx_options& o, LpOutcome& out, std::string& err) {
    return solveTrivialItem(p.item, o, out, err);
}

int32_t solvePrepared(const std::vector<PreparedLp*>& lps, const pdlpx_options& o, const std::atomic<int>* stop,
                      const LpDone& done, std::string& err) {
    const auto t0 = std::chrono::steady_clock::now();
    if (!optionsSupported(o, err)) return PDLPX_E_INVALID;
    std::vector<Item*> items;
    for (PreparedLp* p : lps) {
        if (p->item.trivial) {
            err = "trivial LPs are solved on the host, not in a pack";
            return PDLPX_E_INVALID;
        }
        items.push_back(&p->item);
    }
    if (items.empty()) return PDLPX_OK;
    int32_t rc = selectDevice(o, err);
    if (rc != PDLPX_OK) return rc;
    // the server's packs share the device with each other: no cooperative cycle
    pdlpx_options os = o;
    os.batch_persistent = 0;
    return runPack(items, os, t0, stop, done, err);
}

FamilyPtr makeFamilyBase(const pdlpx_lp& base) {
    auto f = std::make_shared<FamilyBase>();
    Csr a;
    if (base.m <= 0 || base.n <= 0 || base.row_ptr == nullptr ||
        !canonicalCsr(base.m, base.n, base.nnz, base.row_ptr, base.col_idx, base.val, a))
        return nullptr;
    f->m = base.m;
    f->n = base.n;
    f->ptr = std::move(a.ptr);
    f->idx = std::move(a.idx);
    f->val = std::move(a.val);
    return f;
}

bool familyMember(const PreparedLp& p, const FamilyBase& f, const pdlpx_options& o) {
    const HostLp& lp = p.item.lp;
    if (p.item.trivial || o.matrix_zero_tol > 0.0 || f.m <= 0 || lp.n != f.n || lp.m < f.m) return false;
    // gather offsets (index x 32) of the shared rows are int32
    if (static_cast<int64_t>(std::max(f.m, f.n)) * kFamilyLanes >= std::numeric_limits<int32_t>::max()) return false;
    const size_t z = static_cast<size_t>(f.ptr[f.m]);
    return std::equal(f.ptr.begin(), f.ptr.end(), lp.a.ptr.begin()) &&
           std::memcmp(lp.a.idx.data(), f.idx.data(), 4 * z) == 0 &&
           std::memcmp(lp.a.val.data(), f.val.data(), 8 * z) == 0;
}

size_t familyMemberBytes(const PreparedLp& p, const FamilyBase& f) {
    const HostLp& lp = p.item.lp;
    const int64_t extra = lp.m - f.m, zk = lp.a.nnz() - f.ptr[f.m];
    const size_t lane = familyPackBytes(f.n, f.m, 0, 0, 0, famBlocks(f.n), famBlocks(f.m)) / kFam;
    const size_t shared = (24 * static_cast<size_t>(f.ptr[f.m]) + 4 * static_cast<size_t>(f.m + f.n)) / kFam;
    return lane + shared + 120 * static_cast<size_t>(extra) + 28 * static_cast<size_t>(zk);
}

int32_t solveFamily(const FamilyBase& f, const std::vector<PreparedLp*>& lps, const pdlpx_options& o,
                    const std::atomic<int>* stop, const LpDone& done, std::string& err, const FamilyAdmit& admit) {
    const auto t0 = std::chrono::steady_clock::now();
    if (!optionsSupported(o, err)) return PDLPX_E_INVALID;
    if (lps.empty()) return PDLPX_OK;
    if (static_cast<int>(lps.size()) > kFam) {
        err = "a family pack holds at most 32 LPs";
        return PDLPX_E_INVALID;
    }
    FamPack fp;
    fp.base = &f;
    fp.n = f.n;
    fp.mb = f.m;
    for (PreparedLp* p : lps) {
        if (!familyMember(*p, f, o)) {
            err = "LP is not a member of the family (columns or base rows differ)";
            return PDLPX_E_INVALID;
        }
        fp.items.push_back(&p->item);
    }
    fp.L = static_cast<int>(fp.items.size());
    int32_t rc = selectDevice(o, err);
    if (rc != PDLPX_OK) return rc;
    FamAdmit fam_admit;
    if (admit) {
        fam_admit = [&admit](const std::function<bool(const Item&)>& fits, Item*& item, int& id) {
            PreparedLp* p = nullptr;
            if (!admit([&fits](const PreparedLp& q) { return fits(q.item); }, p, id) || p == nullptr) return false;
            item = &p->item;
            return true;
        };
    }
    return solveFamilyPack(fp, o, t0, stop, done, err, fam_admit);
}

int32_t batchSolve(int32_t count, const pdlpx_lp* lps, const pdlpx_options& o, pdlpx_result* results,
                   double* const* x_out, double* const* y_out, std::string& err) {
    const auto t0 = std::chrono::steady_clock::now();
    if (!optionsSupported(o, err)) return PDLPX_E_INVALID;
    std::vector<Item> items(count);
    std::vector<int32_t> codes(count, PDLPX_OK);
    parallelFor(count, [&](int k) { codes[k] = prepareItem(lps[k], o, items[k]); });
    for (int k = 0; k < count; ++k)
        if (codes[k] != PDLPX_OK) {
            err = "invalid LP at index " + std::to_string(k);
            return codes[k];
        }
    auto deliver = [&](int k, LpOutcome& out) {
        results[k] = out.r;
        if (x_out && x_out[k] && !out.x.empty()) std::memcpy(x_out[k], out.x.data(), 8 * out.x.size());
        if (y_out && y_out[k] && !out.y.empty()) std::memcpy(y_out[k], out.y.data(), 8 * out.y.size());
    };
    std::vector<int> dev_items;
    for (int k = 0; k < count; ++k) {
        if (!items[k].trivial) {
            dev_items.push_back(k);
            continue;
        }
        LpOutcome out;
        const int32_t rc = solveTrivialItem(items[k], o, out, err);
        if (rc != PDLPX_OK) return rc;
        deliver(k, out);
    }
    if (dev_items.empty()) return PDLPX_OK;
    int32_t rc = selectDevice(o, err);
    if (rc != PDLPX_OK) return rc;
    size_t free_b = 0, total_b = 0;
    PDLPX_BCK(cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = o.batch_pack_mb > 0 ? static_cast<size_t>(o.batch_pack_mb) << 20
                                              : static_cast<size_t>(0.85 * static_cast<double>(free_b));
    // Packs in input order: a new pack starts when the budget or 32-bit numbering would overflow.
    const int64_t lim32 = std::numeric_limits<int32_t>::max() - 1;
    size_t pos = 0;
    while (pos < dev_items.size()) {
        std::vector<Item*> pack;
        std::vector<int> index;
        size_t bytes = 0;
        int64_t m = 0, n = 0, z = 0, tiles = 0, ent = 0;
        while (pos < dev_items.size()) {
            Item& it = items[dev_items[pos]];
            const int64_t e = std::max(it.cols.entries, it.rows.entries);
            const bool fits = bytes + it.bytes <= budget && m + it.mp < lim32 && n + it.np < lim32 &&
                              z + it.sc.a.nnz() < lim32 && tiles + it.nct + it.nrt < lim32 && ent + e < lim32;
            if (!fits && !pack.empty()) break;
            bytes += it.bytes;
            m += it.mp;
            n += it.np;
            z += it.sc.a.nnz();
            tiles += it.nct + it.nrt;
            ent += e;
            pack.push_back(&it);
            index.push_back(dev_items[pos]);
            ++pos;
        }
        rc = runPack(pack, o, t0, nullptr, [&](int l, LpOutcome&& out) { deliver(index[l], out); }, err);
        if (rc != PDLPX_OK) return rc;
        for (const Item* it : pack)
            if (!it->scale_note.empty()) err = it->scale_note;  // solved; pdlpx_last_error says why scaling was host-side
    }
    return PDLPX_OK;
}

}  // namespace pdlpx

namespace pdlpx {

// Longest-processing-time sharding of independent LPs over ndev devices: the
// heaviest LP first, each onto the device with the least weight assigned so far
// (ties to the lower device index; equal weights keep input order), so the
// assignment is deterministic and no device ends more than one LP's weight
// above the least-loaded one.
void shardLps(int32_t count, const int64_t* weights, int32_t ndev, int32_t* device_of) {
    std::vector<int32_t> order(static_cast<size_t>(count));
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return weights[a] > weights[b]; });
    std::vector<int64_t> load(static_cast<size_t>(ndev), 0);
    for (const int32_t k : order) {
        const int32_t d = static_cast<int32_t>(std::min_element(load.begin(), load.end()) - load.begin());
        device_of[k] = d;
        load[static_cast<size_t>(d)] += weights[k];
    }
}

// pdlpx_batch_solve over several devices: shard by per-iteration work (nonzeros
// + rows + columns), one host thread per device solving its share with the
// single-device batch path (its own stream, packs and budget).  No data moves
// between devices; batch invariance makes every result identical to a
// single-device solve of the same LP.
int32_t batchSolveDevices(int32_t count, const pdlpx_lp* lps, const pdlpx_options& o, const int32_t* devices,
                          int32_t ndev, pdlpx_result* results, double* const* x_out, double* const* y_out,
                          std::string& err) {
    std::vector<int64_t> w(static_cast<size_t>(count));
    for (int32_t k = 0; k < count; ++k)
        w[static_cast<size_t>(k)] = static_cast<int64_t>(lps[k].nnz) + lps[k].m + lps[k].n;
    std::vector<int32_t> dev_of(static_cast<size_t>(count), 0);
    shardLps(count, w.data(), ndev, dev_of.data());
    struct Share {
        std::vector<int32_t> index;
        std::vector<pdlpx_lp> lps;
        std::vector<pdlpx_result> res;
        std::vector<double*> x, y;
        int32_t rc = PDLPX_OK;
        std::string err;
    };
    std::vector<Share> sh(static_cast<size_t>(ndev));
    for (int32_t k = 0; k < count; ++k) {
        Share& s = sh[static_cast<size_t>(dev_of[static_cast<size_t>(k)])];
        s.index.push_back(k);
        s.lps.push_back(lps[k]);
        s.x.push_back(x_out ? x_out[k] : nullptr);
        s.y.push_back(y_out ? y_out[k] : nullptr);
    }
    std::vector<std::thread> th;
    for (int32_t d = 0; d < ndev; ++d) {
        Share& s = sh[static_cast<size_t>(d)];
        if (s.index.empty()) continue;
        s.res.resize(s.index.size());
        th.emplace_back([&s, &o, d, devices] {
            pdlpx_options od = o;
            od.device = devices[d];
            try {
                s.rc = batchSolve(static_cast<int32_t>(s.index.size()), s.lps.data(), od, s.res.data(), s.x.data(),
                                  s.y.data(), s.err);
            } catch (const std::bad_alloc&) {
                s.rc = PDLPX_E_NOMEM;
                s.err = "host allocation failed";
            } catch (const std::exception& e) {
                s.rc = PDLPX_E_INVALID;
                s.err = e.what();
            }
        });
    }
    for (auto& t : th) t.join();
    int32_t rc = PDLPX_OK;
    for (int32_t d = 0; d < ndev; ++d) {
        Share& s = sh[static_cast<size_t>(d)];
        for (size_t i = 0; i < s.index.size() && s.rc == PDLPX_OK; ++i) results[s.index[i]] = s.res[i];
        if (s.rc != PDLPX_OK && rc == PDLPX_OK) {
            rc = s.rc;
            err = "device " + std::to_string(devices[d]) + ": " + s.err;
        } else if (s.rc == PDLPX_OK && !s.err.empty() && err.empty()) {
            err = s.err;  // a note (host-side scaling fallback), not an error
        }
    }
    return rc;
}

// Runs the persistent cycle's grid barrier alone (pdlpx_grid_barrier_check).
// With `stall` the arrival word starts far above any grid size, so no arrival
// completes a barrier: every block polls up to its limit, sets the error word
// and returns, and the call reports PDLPX_E_TIMEOUT with the context intact.
int32_t gridBarrierCheck(int32_t device, int32_t blocks, int32_t rounds, int32_t stall, int32_t* barrier_error,
                         double* seconds, std::string& err) {
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        err = "grid barrier check: no device " + std::to_string(device);
        return PDLPX_E_NO_DEVICE;
    }
    int coop = 0, sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, barrierRounds, 32, 0);
    if (!coop || blocks > per_sm * sms) {
        cudaGetLastError();
        cudaSetDevice(prev);
        err = "grid barrier check: " + std::to_string(blocks) + " blocks do not fit one cooperative wave (" +
              std::to_string(per_sm * sms) + ")";
        return PDLPX_E_INVALID;
    }
    const unsigned preset[4] = {stall ? (1u << 30) : 0u, 0u, 0u, 0u};
    cudaStream_t s = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    unsigned* d = nullptr;
    int h_err = 0;
    float ms = 0.0f;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ev1);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&d), sizeof(preset));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, preset, sizeof(preset), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(ev0, s);
    if (e == cudaSuccess) {
        int r = rounds;
        void* kargs[] = {&d, &r};
        e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&barrierRounds), dim3(blocks), dim3(32), kargs,
                                        0, s);
    }
    if (e == cudaSuccess) e = cudaEventRecord(ev1, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d + 2, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev0, ev1);
    if (e != cudaSuccess) err = std::string("grid barrier check: ") + cudaGetErrorString(e);
    if (s) cudaStreamSynchronize(s);
    if (d) cudaFree(d);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (s) cudaStreamDestroy(s);
    cudaGetLastError();
    cudaSetDevice(prev);
    if (e != cudaSuccess) return PDLPX_E_CUDA;
    *barrier_error = h_err;
    if (seconds) *seconds = ms / 1000.0;
    if (h_err != 0) {
        err = "grid barrier check: a grid barrier ran out of polls";
        return PDLPX_E_TIMEOUT;
    }
    return PDLPX_OK;
}

}  // namespace pdlpx
