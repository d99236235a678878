// Launch-shape dispatch shared by the single-LP engine (engine.cu) and the
// packed batch (batch.cu): compile-time G (lanes per row) and (G, R, U) step
// shapes selected by a runtime index into kShapes.
#pragma once

#include <algorithm>
#include <cstdint>

#include "kernels.cuh"

namespace pdlpx {

#define PDLPX_G_SWITCH(G, CALL)                   \
    switch (G) {                                  \
        case 1: { constexpr int GG = 1; CALL; } break;     \
        case 2: { constexpr int GG = 2; CALL; } break;     \
        case 4: { constexpr int GG = 4; CALL; } break;     \
        case 8: { constexpr int GG = 8; CALL; } break;     \
        case 16: { constexpr int GG = 16; CALL; } break;   \
        case 32: { constexpr int GG = 32; CALL; } break;   \
        case 64: { constexpr int GG = 64; CALL; } break;   \
        case 128: { constexpr int GG = 128; CALL; } break; \
        default: { constexpr int GG = 256; CALL; } break;  \
    }

#define PDLPX_SHAPE_CASE(I, CALL)                                                         \
    case I: {                                                                             \
        constexpr int GG = kShapes[I].G, RR = kShapes[I].R, UU = kShapes[I].U;            \
        CALL;                                                                             \
    } break;
#define PDLPX_SHAPE_SWITCH(S, CALL)                                                                        \
    switch (S) {                                                                                           \
        PDLPX_SHAPE_CASE(0, CALL) PDLPX_SHAPE_CASE(1, CALL) PDLPX_SHAPE_CASE(2, CALL)                      \
        PDLPX_SHAPE_CASE(3, CALL) PDLPX_SHAPE_CASE(4, CALL) PDLPX_SHAPE_CASE(5, CALL)                      \
        PDLPX_SHAPE_CASE(6, CALL) PDLPX_SHAPE_CASE(7, CALL) PDLPX_SHAPE_CASE(8, CALL)                      \
        PDLPX_SHAPE_CASE(9, CALL) PDLPX_SHAPE_CASE(10, CALL) PDLPX_SHAPE_CASE(11, CALL)                    \
        PDLPX_SHAPE_CASE(12, CALL) PDLPX_SHAPE_CASE(13, CALL) PDLPX_SHAPE_CASE(14, CALL)                   \
        default: {                                                                                         \
            constexpr int GG = kShapes[15].G, RR = kShapes[15].R, UU = kShapes[15].U;                      \
            CALL;                                                                                          \
        } break;                                                                                           \
    }
static_assert(kNumShapes == 16, "shape switch covers 16 shapes");

// Shape indices kNumShapes .. kNumShapes + kNumSell - 1 are the sliced-ELL
// variants (one row per thread, kSellU entries per round).
__host__ __device__ constexpr bool isSell(int shape) { return shape >= kNumShapes; }

#define PDLPX_SELL_SWITCH(S, CALL)                                   \
    switch (S - kNumShapes) {                                        \
        case 0: { constexpr int UU = kSellU[0]; CALL; } break;       \
        case 1: { constexpr int UU = kSellU[1]; CALL; } break;       \
        default: { constexpr int UU = kSellU[2]; CALL; } break;      \
    }

// Rows one block of shape `shape` covers.
inline int rowsPerBlock(int shape) { return (kBlock / kShapes[shape].G) * kShapes[shape].R; }

inline int gridForShape(int64_t rows, int shape) {
    const int64_t per_block = rowsPerBlock(shape);
    return static_cast<int>(std::max<int64_t>(1, (rows + per_block - 1) / per_block));
}

// Default launch shape from the mean row length (deterministic; the
// autotuner's starting point).  Picks measured on B200 with FP32 storage: mean
// 2 (1M x 2 transportation A^T) -> G=1; mean 8 -> G=2..4; mean 20 -> G=8;
// mean 1000 (2000 x 1000 transportation A) -> G=64.
inline int defaultShape(int64_t nnz, int32_t rows) {
    const double mean = rows > 0 ? static_cast<double>(nnz) / rows : 0.0;
    if (mean <= 3) return 0;     // G=1
    if (mean <= 6) return 3;     // G=2
    if (mean <= 12) return 5;    // G=4
    if (mean <= 24) return 7;    // G=8
    if (mean <= 48) return 8;    // G=16
    if (mean <= 128) return 9;   // G=32
    return 11;                   // G=64
}

// Default step shape of the packed batch: two rows per lane group so that a
// block of a latency-bound tile keeps twice the loads in flight (measured on
// B200 with 512 lognormal-sized LPs: 4 lanes x 2 rows for mean row lengths 8
// and 20 beat the single-LP table's 4 x 1 and 8 x 1 by 20-30%).
inline int batchShape(int64_t nnz, int32_t rows) {
    const double mean = rows > 0 ? static_cast<double>(nnz) / rows : 0.0;
    if (mean <= 3) return 1;     // G=1, R=2
    if (mean <= 6) return 4;     // G=2, R=2
    if (mean <= 24) return 6;    // G=4, R=2
    if (mean <= 48) return 8;    // G=16
    if (mean <= 128) return 9;   // G=32
    return 11;                   // G=64
}

inline int shapeForGroup(int G) {
    for (int i = 0; i < kNumShapes; ++i)
        if (kShapes[i].G == G && kShapes[i].R == 1) return i;
    return -1;
}

// Step shape of one matrix side from the options: a pinned shape index, else a
// forced lane count, else the row-length table.
inline int chooseShape(int pinned, int group, int64_t nnz, int32_t rows, bool batch = false) {
    if (pinned > 0 && pinned <= kNumShapes) return pinned - 1;
    if (group > 0) {
        const int s = shapeForGroup(group);
        if (s >= 0) return s;
    }
    return batch ? batchShape(nnz, rows) : defaultShape(nnz, rows);
}

}  // namespace pdlpx
