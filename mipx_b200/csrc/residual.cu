// Row-violation reduction of a point against ranged rows, FP64 on the device:
//   v_i = (A x)_i - clamp((A x)_i, row_lb_i, row_ub_i)
//   sum_sq = sum_i v_i^2,  max_abs = max_i |v_i|
// the primal-residual building block of the convergence check
// (pdlp.cpp:1106-1117, pdlp_kernels.cu:280-310).  One G-lane group per row,
// one partial per block in scratch memory, then a single-block pass reduces
// the partials in fixed order, so the result is deterministic.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "engine.hpp"
#include "kernels.cuh"
#include "pdlpx.h"

namespace pdlpx {

template <int G>
__global__ void __launch_bounds__(kBlock) rowViolationKernel(int m, const int* __restrict__ ptr,
                                                            const int* __restrict__ idx,
                                                            const double* __restrict__ val,
                                                            const double* __restrict__ x,
                                                            const double* __restrict__ rl,
                                                            const double* __restrict__ ru, double* partials) {
    const int t = blockIdx.x * kBlock + threadIdx.x;
    const int i = t / G, lane = t % G;
    const bool valid = i < m;
    double s = 0.0;
    if (valid) s = rowDotU<G, 4, double>(ptr[i], ptr[i + 1], lane, idx, val, x);
    s = groupSum<G>(s);
    double acc[2] = {0.0, 0.0};
    if (valid && lane == 0) {
        const double lo = rl[i], hi = ru[i];
        const double c = s < lo ? lo : (hi < s ? hi : s);
        const double v = s - c;
        acc[0] = v * v;
        acc[1] = fabs(v);
    }
    const int ops[2] = {OP_SUM, OP_MAX};
    blockReduceSlots<2>(acc, ops, partials + static_cast<size_t>(blockIdx.x) * 2);
}

__global__ void __launch_bounds__(kBlock) rowViolationFinish(int nb, const double* partials, double* out) {
    double acc[2] = {0.0, 0.0};
    for (int b = threadIdx.x; b < nb; b += kBlock) {
        acc[0] += partials[static_cast<size_t>(b) * 2];
        acc[1] = fmax(acc[1], partials[static_cast<size_t>(b) * 2 + 1]);
    }
    __shared__ double res[2];
    const int ops[2] = {OP_SUM, OP_MAX};
    blockReduceSlots<2>(acc, ops, res);
    __syncthreads();
    if (threadIdx.x < 2) out[threadIdx.x] = res[threadIdx.x];
}

// Number of blocks of the row kernel for m rows at G lanes per row.
static int rowViolationBlocks(int64_t m, int G) {
    return static_cast<int>(std::max<int64_t>(1, (m * G + kBlock - 1) / kBlock));
}

// Enqueue both kernels on `stream`; partials must hold 2 * blocks doubles.
static cudaError_t launchRowViolation(int m, int G, const int* ptr, const int* idx, const double* val,
                                      const double* x, const double* rl, const double* ru, double* partials,
                                      double* out, cudaStream_t stream) {
    const int nb = rowViolationBlocks(m, G);
    switch (G) {
        case 1: rowViolationKernel<1><<<nb, kBlock, 0, stream>>>(m, ptr, idx, val, x, rl, ru, partials); break;
        case 2: rowViolationKernel<2><<<nb, kBlock, 0, stream>>>(m, ptr, idx, val, x, rl, ru, partials); break;
        case 4: rowViolationKernel<4><<<nb, kBlock, 0, stream>>>(m, ptr, idx, val, x, rl, ru, partials); break;
        case 8: rowViolationKernel<8><<<nb, kBlock, 0, stream>>>(m, ptr, idx, val, x, rl, ru, partials); break;
        case 16: rowViolationKernel<16><<<nb, kBlock, 0, stream>>>(m, ptr, idx, val, x, rl, ru, partials); break;
        case 32: rowViolationKernel<32><<<nb, kBlock, 0, stream>>>(m, ptr, idx, val, x, rl, ru, partials); break;
        case 64: rowViolationKernel<64><<<nb, kBlock, 0, stream>>>(m, ptr, idx, val, x, rl, ru, partials); break;
        case 128: rowViolationKernel<128><<<nb, kBlock, 0, stream>>>(m, ptr, idx, val, x, rl, ru, partials); break;
        default: rowViolationKernel<256><<<nb, kBlock, 0, stream>>>(m, ptr, idx, val, x, rl, ru, partials); break;
    }
    rowViolationFinish<<<1, kBlock, 0, stream>>>(nb, partials, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free variant.  Some callers cannot call cudaMalloc: code running
// inside another framework's memory pool, or under a graph or allocator policy
// that forbids new device allocations.  For them the per-block partials of the
// row kernel live in this fixed device array instead of a cudaMalloc'd buffer.
// Every GPU that loads this library holds the array (64 KiB) until the process
// exits.  All calls on a device share it and it keeps the last call's contents;
// every block writes its own partial before the final pass reads it, so nothing
// needs clearing, but calls that overlap on the GPU race on it.
// ---------------------------------------------------------------------------
constexpr int kNoAllocBlocks = 4096;  // at most 4096 row blocks of 256 threads per call
static __device__ __align__(256) double g_row_violation_scratch[2 * kNoAllocBlocks];

namespace {
std::mutex g_scratch_mutex;
constexpr int kMaxDevices = 256;
double* g_scratch_address[kMaxDevices] = {};  // device address of the array, per device
}  // namespace

}  // namespace pdlpx

using namespace pdlpx;

extern "C" {

int32_t pdlpx_row_violation(int32_t m, int32_t n, int32_t nnz, const int32_t* row_ptr, const int32_t* col_idx,
                            const double* val, const double* x, const double* row_lb, const double* row_ub,
                            double* sum_sq, double* max_abs) {
    if (m < 0 || n < 0 || nnz < 0 || sum_sq == nullptr || max_abs == nullptr ||
        (m > 0 && (row_ptr == nullptr || row_lb == nullptr || row_ub == nullptr)) ||
        (nnz > 0 && (col_idx == nullptr || val == nullptr)) || (n > 0 && x == nullptr))
        return PDLPX_E_INVALID;
    *sum_sq = 0.0;
    *max_abs = 0.0;
    if (m == 0) return PDLPX_OK;
    if (row_ptr[0] != 0 || row_ptr[m] != nnz) return PDLPX_E_INVALID;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) return PDLPX_E_NO_DEVICE;
    const int G = pickGroup(nnz, m);
    const int nb = rowViolationBlocks(m, G);
    auto al = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
    const size_t o_ptr = 0, o_idx = o_ptr + al(4 * (static_cast<size_t>(m) + 1)),
                 o_val = o_idx + al(4 * static_cast<size_t>(nnz)), o_x = o_val + al(8 * static_cast<size_t>(nnz)),
                 o_rl = o_x + al(8 * static_cast<size_t>(std::max(n, 1))), o_ru = o_rl + al(8 * static_cast<size_t>(m)),
                 o_part = o_ru + al(8 * static_cast<size_t>(m)), o_out = o_part + al(16 * static_cast<size_t>(nb)),
                 total = o_out + 16;
    char* buf = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(&buf), total) != cudaSuccess) return PDLPX_E_NOMEM;
    struct Free {
        char* p;
        ~Free() { cudaFree(p); }
    } guard{buf};
    cudaError_t e = cudaSuccess;
    auto up = [&](size_t off, const void* src, size_t bytes) {
        if (e == cudaSuccess && bytes > 0) e = cudaMemcpy(buf + off, src, bytes, cudaMemcpyHostToDevice);
    };
    up(o_ptr, row_ptr, 4 * (static_cast<size_t>(m) + 1));
    up(o_idx, col_idx, 4 * static_cast<size_t>(nnz));
    up(o_val, val, 8 * static_cast<size_t>(nnz));
    up(o_x, x, 8 * static_cast<size_t>(n));
    up(o_rl, row_lb, 8 * static_cast<size_t>(m));
    up(o_ru, row_ub, 8 * static_cast<size_t>(m));
    if (e != cudaSuccess) return PDLPX_E_CUDA;
    e = launchRowViolation(m, G, reinterpret_cast<int*>(buf + o_ptr), reinterpret_cast<int*>(buf + o_idx),
                           reinterpret_cast<double*>(buf + o_val), reinterpret_cast<double*>(buf + o_x),
                           reinterpret_cast<double*>(buf + o_rl), reinterpret_cast<double*>(buf + o_ru),
                           reinterpret_cast<double*>(buf + o_part), reinterpret_cast<double*>(buf + o_out), nullptr);
    if (e != cudaSuccess) return PDLPX_E_CUDA;
    double out[2];
    if (cudaMemcpy(out, buf + o_out, 16, cudaMemcpyDeviceToHost) != cudaSuccess) return PDLPX_E_CUDA;
    *sum_sq = out[0];
    *max_abs = out[1];
    return PDLPX_OK;
}

int32_t pdlpx_row_violation_noalloc(int32_t m, int32_t n, int32_t nnz, const int32_t* d_row_ptr,
                                    const int32_t* d_col_idx, const double* d_val, const double* d_x,
                                    const double* d_row_lb, const double* d_row_ub, double* d_out, void* stream) {
    try {
    if (m < 0 || n < 0 || nnz < 0 || d_out == nullptr ||
        (m > 0 && (d_row_ptr == nullptr || d_row_lb == nullptr || d_row_ub == nullptr)) ||
        (nnz > 0 && (d_col_idx == nullptr || d_val == nullptr)) || (n > 0 && d_x == nullptr)) {
        setGlobalError("pdlpx_row_violation_noalloc: invalid argument");
        return PDLPX_E_INVALID;
    }
    const int G = pickGroup(nnz, m);
    const int nb = rowViolationBlocks(m, G);
    if (nb > kNoAllocBlocks) {
        setGlobalError("pdlpx_row_violation_noalloc: " + std::to_string(m) + " rows at " + std::to_string(G) +
                       " threads per row need " + std::to_string(nb) + " blocks; the fixed scratch holds " +
                       std::to_string(kNoAllocBlocks) + " (m * G <= 1048576)");
        return PDLPX_E_INVALID;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        setGlobalError("pdlpx_row_violation_noalloc: no current CUDA device");
        return PDLPX_E_NO_DEVICE;
    }
    double* scratch = nullptr;
    {
        // One-time set-up per device, with that device current: resolve the
        // array's device address (host code cannot use the symbol itself).
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (g_scratch_address[dev] == nullptr) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_row_violation_scratch);
            if (e != cudaSuccess || p == nullptr) {
                setGlobalError(std::string("pdlpx_row_violation_noalloc: cudaGetSymbolAddress failed: ") +
                               cudaGetErrorString(e));
                return PDLPX_E_CUDA;
            }
            g_scratch_address[dev] = static_cast<double*>(p);
        }
        scratch = g_scratch_address[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (m == 0) {
        return cudaMemsetAsync(d_out, 0, 2 * sizeof(double), s) == cudaSuccess ? PDLPX_OK : PDLPX_E_CUDA;
    }
    const cudaError_t e =
        launchRowViolation(m, G, d_row_ptr, d_col_idx, d_val, d_x, d_row_lb, d_row_ub, scratch, d_out, s);
    if (e != cudaSuccess) {
        setGlobalError(std::string("pdlpx_row_violation_noalloc: launch failed: ") + cudaGetErrorString(e));
        return PDLPX_E_CUDA;
    }
    return PDLPX_OK;
    } catch (const std::bad_alloc&) {
        return PDLPX_E_NOMEM;  // building an error message failed; nothing was enqueued
    } catch (...) {
        return PDLPX_E_INVALID;
    }
}

}  // extern "C"
