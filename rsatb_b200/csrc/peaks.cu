// Measured FMA-pipe peak (FP64, FP32, FP32 issued as packed f32x2 FMAs,
// FP64 on the tensor cores as m8n8k4 tiles, or TF32 on the tensor cores as
// mma.sync m16n8k8 tiles),
// the denominator of the compute roofline of the SpMM at wide panels, where
// the block SpMM is bound by the CUDA-core FMA rate rather than by HBM.
// Every SM runs independent FMA chains; the result is FLOP/s = 2 * FMAs /
// elapsed time (CUDA events).
#include "common.cuh"

namespace rsatb_b200 {
namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_chains(T* out, int iters, T a, T b) {
    T x0 = T(threadIdx.x) * T(1e-3), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
    T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == T(-12345.678)) out[threadIdx.x] = s;  // keeps the chains live
}

// Eight chains of packed pairs: fma.rn.f32x2 (sm_100) does two FP32 FMAs.
__global__ void __launch_bounds__(256) fma2_chains(float* out, int iters, float a, float b) {
    unsigned long long x[8];
    const float base = float(threadIdx.x) * 1e-3f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float lo = base + float(2 * k), hi = base + float(2 * k + 1);
        asm("mov.b64 %0, {%1, %2};" : "=l"(x[k]) : "f"(lo), "f"(hi));
    }
    unsigned long long av, bv;
    asm("mov.b64 %0, {%1, %1};" : "=l"(av) : "f"(a));
    asm("mov.b64 %0, {%1, %1};" : "=l"(bv) : "f"(b));
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int k = 0; k < 8; ++k)
                asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[k]) : "l"(av), "l"(bv));
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float lo, hi;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x[k]));
        s += lo + hi;
    }
    if (s == -12345.678f) out[threadIdx.x] = s;  // keeps the chains live
}

// Eight independent chains of FP64 tensor-core tiles (mma.sync m8n8k4 f64:
// 256 FMAs per warp per instruction).
__global__ void __launch_bounds__(256) dmma_chains(double* out, int iters, double a, double b) {
    double d[8][2];
#pragma unroll
    for (int k = 0; k < 8; ++k) d[k][0] = d[k][1] = double(threadIdx.x) * 1e-3 + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int k = 0; k < 8; ++k)
                asm volatile(
                    "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, "
                    "{%0, %1};"
                    : "+d"(d[k][0]), "+d"(d[k][1])
                    : "d"(a), "d"(b));
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += d[k][0] + d[k][1];
    if (s == -12345.678) out[threadIdx.x] = s;  // keeps the chains live
}

// Eight independent chains of TF32 tensor-core tiles (mma.sync m16n8k8
// tf32 with FP32 accumulation: 1024 FMAs per warp per instruction).
__global__ void __launch_bounds__(256) tf32_mma_chains(float* out, int iters, float a, float b) {
    float d[8][4];
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int e = 0; e < 4; ++e) d[k][e] = float(threadIdx.x) * 1e-3f + float(k + e);
    const uint32_t av = __float_as_uint(a), bv = __float_as_uint(b);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int k = 0; k < 8; ++k)
                asm volatile(
                    "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, "
                    "{%4, %4, %4, %4}, {%5, %5}, {%0, %1, %2, %3};"
                    : "+f"(d[k][0]), "+f"(d[k][1]), "+f"(d[k][2]), "+f"(d[k][3])
                    : "r"(av), "r"(bv));
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += d[k][0] + d[k][1] + d[k][2] + d[k][3];
    if (s == -12345.678f) out[threadIdx.x] = s;  // keeps the chains live
}

}  // namespace
}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" int rsatb_measure_fma_peak(rsatb_ctx_t ctx, int double_precision, double* flops) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!flops) return set_error(RSATB_INVALID_ARGUMENT, "null output");
    void* sink = nullptr;
    RSATB_TRY(ctx_scratch(ctx, 4096, &sink));
    const int threads = 256;
    const int grid = ctx->sm_count * 8;
    if (double_precision < 0 || double_precision > 4)
        return set_error(RSATB_INVALID_ARGUMENT, "unknown peak kind %d", double_precision);
    const int iters = double_precision == 1 ? 4096
                      : (double_precision == 3 || double_precision == 4) ? 64 : 8192;
    cudaEvent_t e0, e1;
    RSATB_CUDA_TRY(cudaEventCreate(&e0));
    RSATB_CUDA_TRY(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        RSATB_CUDA_TRY(cudaEventRecord(e0, ctx->stream));
        if (double_precision == 4)
            tf32_mma_chains<<<grid, threads, 0, ctx->stream>>>((float*)sink, iters, 1e-3f, 1e-3f);
        else if (double_precision == 3)
            dmma_chains<<<grid, threads, 0, ctx->stream>>>((double*)sink, iters, 0.999999, 1e-7);
        else if (double_precision == 2)
            fma2_chains<<<grid, threads, 0, ctx->stream>>>((float*)sink, iters, 0.9999f, 1e-4f);
        else if (double_precision)
            fma_chains<double><<<grid, threads, 0, ctx->stream>>>((double*)sink, iters,
                                                                   0.999999, 1e-7);
        else
            fma_chains<float><<<grid, threads, 0, ctx->stream>>>((float*)sink, iters, 0.9999f,
                                                                  1e-4f);
        RSATB_LAUNCH_CHECK(ctx);
        RSATB_CUDA_TRY(cudaEventRecord(e1, ctx->stream));
        RSATB_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        RSATB_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0 && ms < best_ms) best_ms = ms;  // first run warms up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // Per thread and inner step: 1 FMA (scalar), 2 (f32x2), 256 / 32 = 8
    // (one m8n8k4 tile per warp) or 1024 / 32 = 32 (one m16n8k8 tile).
    const double per = double_precision == 2 ? 2.0
                       : double_precision == 3 ? 8.0
                       : double_precision == 4 ? 32.0 : 1.0;
    const double fmas = double(grid) * threads * double(iters) * 4.0 * 8.0 * per;
    *flops = 2.0 * fmas / (double(best_ms) * 1e-3);
    return RSATB_SUCCESS;
}
