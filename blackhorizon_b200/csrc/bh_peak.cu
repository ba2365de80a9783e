// bh_peak.cu -- vector FMA throughput probe: the FP32 / FP64 CUDA-core peak
// that the tracer kernels' roofline fraction is quoted against (the tensor
// cores do not apply to this path).
#include "bh_internal.h"

namespace bh {

// 8 independent FMA chains per thread keep every FMA pipe busy; the result
// is folded into one store so the compiler keeps the work.
template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(long long iters, T *sink) {
    T a0 = T(threadIdx.x) * T(1e-3), a1 = a0 + T(1), a2 = a0 + T(2), a3 = a0 + T(3);
    T a4 = a0 + T(4), a5 = a0 + T(5), a6 = a0 + T(6), a7 = a0 + T(7);
    const T m = T(0.999999), c = T(1e-7);
    for (long long i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
            a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
        }
    }
    const T s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == T(-1)) sink[0] = s;  // never true; keeps the chains live
}

// The same with packed float32x2 FMAs (sm_100 FFMA2): 8 chains of two lanes.
__global__ void __launch_bounds__(256) fma2_peak_kernel(long long iters, float *sink) {
    const float b = float(threadIdx.x) * 1e-3f;
    float2 a0 = make_float2(b, b + 0.5f), a1 = make_float2(b + 1, b + 1.5f);
    float2 a2 = make_float2(b + 2, b + 2.5f), a3 = make_float2(b + 3, b + 3.5f);
    float2 a4 = make_float2(b + 4, b + 4.5f), a5 = make_float2(b + 5, b + 5.5f);
    float2 a6 = make_float2(b + 6, b + 6.5f), a7 = make_float2(b + 7, b + 7.5f);
    const float2 m = make_float2(0.999999f, 0.999999f), c = make_float2(1e-7f, 1e-7f);
    for (long long i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = __ffma2_rn(a0, m, c); a1 = __ffma2_rn(a1, m, c);
            a2 = __ffma2_rn(a2, m, c); a3 = __ffma2_rn(a3, m, c);
            a4 = __ffma2_rn(a4, m, c); a5 = __ffma2_rn(a5, m, c);
            a6 = __ffma2_rn(a6, m, c); a7 = __ffma2_rn(a7, m, c);
        }
    }
    const float s = ((a0.x + a1.x) + (a2.x + a3.x)) + ((a4.y + a5.y) + (a6.y + a7.y));
    if (s == -1.0f) sink[0] = s;
}

}  // namespace bh

extern "C" int bh_fma_peak_launch(int32_t precision, int64_t iters, void *sink,
                                  int64_t *flops, void *stream) {
    using namespace bh;
    if (iters < 1 || !sink || !flops) return BH_ERR_INVALID_ARGUMENT;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        set_error("bh_fma_peak_launch: no device");
        return BH_ERR_CUDA;
    }
    const int block = 256;
    const int blocks = sms * 8;
    if (precision == BH_PRECISION_FP64) {
        fma_peak_kernel<double><<<blocks, block, 0, (cudaStream_t)stream>>>(iters, (double *)sink);
        *flops = (int64_t)blocks * block * iters * 16 * 8 * 2;
    } else if (precision == BH_PEAK_F32X2) {
        fma2_peak_kernel<<<blocks, block, 0, (cudaStream_t)stream>>>(iters, (float *)sink);
        *flops = (int64_t)blocks * block * iters * 16 * 8 * 4;
    } else {
        fma_peak_kernel<float><<<blocks, block, 0, (cudaStream_t)stream>>>(iters, (float *)sink);
        *flops = (int64_t)blocks * block * iters * 16 * 8 * 2;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("bh_fma_peak_launch: %s", cudaGetErrorString(e));
        return BH_ERR_CUDA;
    }
    return BH_OK;
}
