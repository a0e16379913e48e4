// bh_peak.cu -- FMA throughput microkernels (no counterpart in the
// reference): the FP64 and FP32 pipe peaks that bound the compute-heavy
// stencil kernels, measured on the device the library runs on.
#include <cuda_runtime.h>
#include <stdint.h>
#include "bhgpu.h"

namespace {
constexpr int PEAK_TPB = 256;
// CH independent multiply-add chains per thread keep the pipe busy; the
// values stay finite (a fixed point of a -> a c + d with c < 1)
template <typename T, int CH>
__global__ void __launch_bounds__(PEAK_TPB) k_peak(T* out, int64_t n, int iters, T c, T d) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    T a[CH];
#pragma unroll
    for (int k = 0; k < CH; k++) a[k] = T(t % 97) * T(0.01) + T(k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < CH; k++) a[k] = fma(a[k], c, d);
    }
    T s = T(0);
#pragma unroll
    for (int k = 0; k < CH; k++) s += a[k];
    if (t < n) out[t] = s;
}
}  // namespace

extern "C" int bh_peak_fma(int32_t precision, int32_t iters, void* out, int64_t n, int64_t* flops, void* stream) {
    if (!out || n <= 0 || iters <= 0 || !flops) return BH_EINVAL;
    const int64_t blocks = (n + PEAK_TPB - 1) / PEAK_TPB;
    cudaStream_t s = (cudaStream_t)stream;
    if (precision == BH_FP64) {
        constexpr int CH = 8;
        k_peak<double, CH><<<(unsigned)blocks, PEAK_TPB, 0, s>>>((double*)out, n, iters, 0.999999, 1e-6);
        *flops = 2 * (int64_t)CH * iters * blocks * PEAK_TPB;
    } else if (precision == BH_MIXED) {
        constexpr int CH = 16;
        k_peak<float, CH><<<(unsigned)blocks, PEAK_TPB, 0, s>>>((float*)out, n, iters, 0.999f, 1e-3f);
        *flops = 2 * (int64_t)CH * iters * blocks * PEAK_TPB;
    } else {
        return BH_EINVAL;
    }
    return cudaGetLastError() == cudaSuccess ? BH_OK : BH_ECUDA;
}
