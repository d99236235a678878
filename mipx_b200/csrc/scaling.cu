// Ruiz equilibration on the device (the O(passes x nnz) part of the scaling
// pipeline, pdlp.cpp:520-558).
//
// Each pass scales every row by 1/sqrt(max_k |a_ik|) (rows whose max is at or
// below 1e-12 are left alone), then every column by 1/sqrt of its max over the
// row-scaled values, accumulating the factors in row_scale / col_scale.  The
// operations per entry are the host pipeline's own -- one correctly rounded
// sqrt, one division, one multiply each -- and a max does not depend on the
// order it is taken in, so the scaled matrix and both scale vectors are
// bit-identical to the host's (buildScaled in problem.cpp).  The column max is
// an atomic max on the bit pattern of |a| (non-negative doubles order like
// their bits).  The rest of the pipeline (cost and bound scaling,
// Pock-Chambolle, bound/objective rescaling, the transpose) stays on the host.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "problem.hpp"

namespace pdlpx {
namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) ruizRows(int m, const int* __restrict__ ptr, double* __restrict__ val,
                                                      double* __restrict__ rs) {
    const int i = blockIdx.x * (kThreads / 32) + static_cast<int>(threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= m) return;
    const int b = ptr[i], e = ptr[i + 1];
    double mx = 0.0;
    for (int k = b + lane; k < e; k += 32) mx = fmax(mx, fabs(val[k]));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if (mx <= 1e-12) return;
    const double f = 1.0 / sqrt(mx);
    if (lane == 0) rs[i] *= f;
    for (int k = b + lane; k < e; k += 32) val[k] *= f;
}

__global__ void __launch_bounds__(kThreads) ruizColMax(int64_t nnz, const int* __restrict__ idx,
                                                        const double* __restrict__ val,
                                                        unsigned long long* __restrict__ cmax) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(kThreads) + threadIdx.x; k < nnz;
         k += static_cast<int64_t>(gridDim.x) * kThreads)
        atomicMax(cmax + idx[k], static_cast<unsigned long long>(__double_as_longlong(fabs(val[k]))));
}

__global__ void __launch_bounds__(kThreads) ruizCols(int n, int64_t nnz, const int* __restrict__ idx,
                                                      double* __restrict__ val,
                                                      const unsigned long long* __restrict__ cmax,
                                                      double* __restrict__ cs) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * kThreads;
    for (int64_t j = blockIdx.x * static_cast<int64_t>(kThreads) + threadIdx.x; j < n; j += stride) {
        const double cm = __longlong_as_double(static_cast<long long>(cmax[j]));
        if (cm > 1e-12) cs[j] *= 1.0 / sqrt(cm);
    }
    for (int64_t k = blockIdx.x * static_cast<int64_t>(kThreads) + threadIdx.x; k < nnz; k += stride) {
        const double cm = __longlong_as_double(static_cast<long long>(cmax[idx[k]]));
        if (cm > 1e-12) val[k] *= 1.0 / sqrt(cm);
    }
}

}  // namespace

bool ruizOnDevice(Csr& a, std::vector<double>& row_scale, std::vector<double>& col_scale, int passes, int device,
                  std::string& err, bool verbose) {
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    const int m = a.rows, n = a.cols;
    const int64_t nnz = a.nnz();
    if (m <= 0 || n <= 0 || nnz <= 0 || passes <= 0) return true;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        err = "device scaling: no such device";
        return false;
    }
    cudaStream_t s = nullptr;
    char* d = nullptr;
    auto fail = [&](cudaError_t e, const char* what) {
        err = std::string("device scaling: ") + what + ": " + cudaGetErrorString(e);
        if (d) cudaFreeAsync(d, s);
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
        cudaGetLastError();
        cudaSetDevice(prev);
        return false;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(e, "stream");
    auto al = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
    const size_t o_ptr = 0, o_idx = o_ptr + al(4 * (static_cast<size_t>(m) + 1)),
                 o_val = o_idx + al(4 * static_cast<size_t>(nnz)), o_rs = o_val + al(8 * static_cast<size_t>(nnz)),
                 o_cs = o_rs + al(8 * static_cast<size_t>(m)), o_cm = o_cs + al(8 * static_cast<size_t>(n)),
                 total = o_cm + al(8 * static_cast<size_t>(n));
    if ((e = cudaMallocAsync(reinterpret_cast<void**>(&d), total, s)) != cudaSuccess) return fail(e, "allocation");
    int* ptr = reinterpret_cast<int*>(d + o_ptr);
    int* idx = reinterpret_cast<int*>(d + o_idx);
    double* val = reinterpret_cast<double*>(d + o_val);
    double* rs = reinterpret_cast<double*>(d + o_rs);
    double* cs = reinterpret_cast<double*>(d + o_cs);
    auto* cm = reinterpret_cast<unsigned long long*>(d + o_cm);
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice, d2h = cudaMemcpyDeviceToHost;
    if ((e = cudaMemcpyAsync(ptr, a.ptr.data(), 4 * (static_cast<size_t>(m) + 1), h2d, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(idx, a.idx.data(), 4 * static_cast<size_t>(nnz), h2d, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(val, a.val.data(), 8 * static_cast<size_t>(nnz), h2d, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(rs, row_scale.data(), 8 * static_cast<size_t>(m), h2d, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(cs, col_scale.data(), 8 * static_cast<size_t>(n), h2d, s)) != cudaSuccess)
        return fail(e, "upload");
    const auto t1 = clk::now();
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int grow = static_cast<int>((static_cast<int64_t>(m) + kThreads / 32 - 1) / (kThreads / 32));
    const int gent = static_cast<int>(std::min<int64_t>((nnz + kThreads - 1) / kThreads, 8LL * sms));
    for (int pass = 0; pass < passes; ++pass) {
        ruizRows<<<grow, kThreads, 0, s>>>(m, ptr, val, rs);
        cudaMemsetAsync(cm, 0, 8 * static_cast<size_t>(n), s);
        ruizColMax<<<gent, kThreads, 0, s>>>(nnz, idx, val, cm);
        ruizCols<<<gent, kThreads, 0, s>>>(n, nnz, idx, val, cm, cs);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "launch");
    if (verbose && (e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e, "synchronize");
    const auto t2 = clk::now();
    // read back into the caller's arrays (already touched memory: no page
    // faults during the copy); a failure from here on leaves them partly
    // written, and the caller restarts from the unscaled values
    if ((e = cudaMemcpyAsync(a.val.data(), val, 8 * static_cast<size_t>(nnz), d2h, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(row_scale.data(), rs, 8 * static_cast<size_t>(m), d2h, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(col_scale.data(), cs, 8 * static_cast<size_t>(n), d2h, s)) != cudaSuccess)
        return fail(e, "read back");
    cudaFreeAsync(d, s);
    d = nullptr;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e, "synchronize");
    cudaStreamDestroy(s);
    cudaSetDevice(prev);
    if (verbose) {
        auto sec = [](clk::time_point x, clk::time_point y) { return std::chrono::duration<double>(y - x).count(); };
        std::printf("PDLP device Ruiz: set-up + upload %.3fs, %d passes %.3fs, read back %.3fs\n", sec(t0, t1), passes,
                    sec(t1, t2), sec(t2, clk::now()));
        std::fflush(stdout);
    }
    return true;
}

RuizFn ruizFor(const pdlpx_options& o, int64_t nnz, std::string* fallback_note) {
    if (!(o.scale_on_device > 0 || (o.scale_on_device < 0 && nnz >= 200000))) return {};
    const int device = o.device;
    const bool verbose = o.verbose != 0;
    return [device, verbose, fallback_note](Csr& a, std::vector<double>& rs, std::vector<double>& cs, int passes) {
        std::string err;
        const bool ok = ruizOnDevice(a, rs, cs, passes, device, err, verbose);
        if (!ok && fallback_note != nullptr) *fallback_note = "device Ruiz scaling fell back to the host: " + err;
        return ok;
    };
}

}  // namespace pdlpx
