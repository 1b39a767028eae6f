// Fused Chebyshev step on the FP64 tensor cores: real 8x8 blocks, panels of
// W = 8 to 256 real values per row (W a multiple of 8), stored in FP64 or
// FP32 (VT).  FP32 operands are widened to FP64 as they are loaded, so an
// FP32 panel is multiplied with FP64 products and FP64 accumulation (its
// result is rounded to FP32 once, at the store).
//
// An 8x8 block times 8 panel columns is exactly two mma.sync m8n8k4 f64
// tiles (K = 8 split in two halves of 4): the block is the A operand (one
// value per lane at row lane / 4, column lane % 4 + 4h) and 8 columns of the
// gathered X_j rows the B operand (one value per lane at row lane % 4 + 4h,
// column lane / 4).  A warp owns one block row and all W / 8 column groups,
// so each of its fragment loads is a warp-wide read (8 rows x 32 bytes of A;
// for X_j of an FP64 panel with W a multiple of 16, 4 rows x 128 bytes: two column
// groups take the even and the odd columns of a 16-column span, so one
// 2-value load per lane feeds two fragments) and each MMA instruction
// carries 256 FMAs.  For narrow panels U blocks of the row are loaded together, so
// several blocks are in flight per warp.
//
// The accumulator leaves each lane two (four, paired) consecutive columns
// of one output row per column group (pair), which is the layout finish_row
// expects with V = 2 (4); the (re, im) pairs of a complex panel stay
// together.  The FP64 column
// dots of the epilogue are summed over the block row's 8 rows by shuffles
// and accumulated per warp in shared memory; the CTA then sums its warps in
// a fixed order and finish_partials sums the CTAs (deterministic).
#pragma once

#include "cheb_kernels.cuh"

namespace rsatb_b200 {

// Warps per CTA: 8 for FP32 panels (neighbouring block rows of one CTA
// share their gathered X_j lines in L1: FP32 R = 8 0.080 -> 0.062 ms on the
// diamond 8x8 BSR), 4 for FP64 (more warps measured slower at R = 128).
template <typename VT>
constexpr int dmma_warps() {
    return sizeof(VT) == 4 ? 8 : 4;
}

__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Blocks of a row loaded together (UU, 0: by width): enough loads in flight
// at narrow panels, registers bounded at wide ones.
template <int W, int UU = 0>
struct DmmaShape {
    static constexpr int NG = W / 8;
    static constexpr int U = UU ? UU : (W <= 16 ? 4 : (W <= 32 ? 2 : 1));
};

template <typename VT, int W, bool CV, int UU>
__global__ void __launch_bounds__(dmma_warps<VT>() * 32) cheb_step_dmma(StepArgs a) {
    constexpr int kDmmaWarps = dmma_warps<VT>();
    static_assert(W % 8 == 0 && W <= 256, "8-column groups");
    constexpr int NG = DmmaShape<W, UU>::NG, U = DmmaShape<W, UU>::U;
    // 16-column spans with 2-value X loads: FP64 panels (measured at FP32
    // W = 16 the single-value loads are faster).
    constexpr bool PAIRED = NG % 2 == 0 && sizeof(VT) == 8;
    __shared__ double dsm[kDmmaWarps][2][W];  // per warp: dots d0, d1 per column
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int fr = lane >> 2, fc = lane & 3;
    const VT* __restrict__ vals = static_cast<const VT*>(a.vals);
    const VT* __restrict__ in = static_cast<const VT*>(a.in);
    const int ndots = a.dot_mode == DOT_DOUBLING ? 2 : (a.dot_mode == DOT_PLAIN ? 1 : 0);
    for (int c = lane; c < 2 * W; c += 32) dsm[warp][c / W][c % W] = 0.0;
    __syncwarp();

    for (int64_t i = int64_t(blockIdx.x) * kDmmaWarps + warp; i < a.n_block_rows;
         i += int64_t(gridDim.x) * kDmmaWarps) {
        const int k0 = __ldg(a.row_ptr + i), k1 = __ldg(a.row_ptr + i + 1);
        double acc[NG][2];
#pragma unroll
        for (int g = 0; g < NG; ++g) acc[g][0] = acc[g][1] = 0.0;
        for (int k = k0; k < k1; k += U) {
            double af[U][2], bf[U][NG][2];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int kk = k + u;
                const bool valid = kk < k1;
                const int64_t j = valid ? __ldg(a.col_ind + kk) : 0;
                const VT* blk = vals + int64_t(valid ? kk : k0) * 64 + fr * 8 + fc;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    af[u][h] = valid ? double(__ldg(blk + 4 * h)) : 0.0;
                    if constexpr (PAIRED) {
                        // Groups 2p and 2p + 1 take the even and the odd
                        // columns of the 16-column span 16p..16p + 15: one
                        // 2-value load per lane feeds both fragments.
                        const VT* xr = in + (j * 8 + fc + 4 * h) * W + 2 * fr;
#pragma unroll
                        for (int p = 0; p < NG / 2; ++p) {
                            double e = 0.0, o = 0.0;
                            if (valid) {
                                if constexpr (sizeof(VT) == 8) {
                                    const double2 t = __ldg(reinterpret_cast<const double2*>(xr + 16 * p));
                                    e = t.x;
                                    o = t.y;
                                } else {
                                    const float2 t = __ldg(reinterpret_cast<const float2*>(xr + 16 * p));
                                    e = t.x;
                                    o = t.y;
                                }
                            }
                            bf[u][2 * p][h] = e;
                            bf[u][2 * p + 1][h] = o;
                        }
                    } else {
                        const VT* xr = in + (j * 8 + fc + 4 * h) * W + fr;
#pragma unroll
                        for (int g = 0; g < NG; ++g)
                            bf[u][g][h] = valid ? double(__ldg(xr + 8 * g)) : 0.0;
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int h = 0; h < 2; ++h)
#pragma unroll
                    for (int g = 0; g < NG; ++g) dmma_884(acc[g], af[u][h], bf[u][g][h]);
        }
        // Epilogue.  Unpaired: lane holds output row i*8 + fr, columns
        // 8g + 2fc + {0, 1} of group g.  Paired: groups 2p, 2p + 1 give it
        // columns 16p + 4fc + {0, 1, 2, 3} (even fragment first).
        constexpr int VE = PAIRED ? 4 : 2;
#pragma unroll
        for (int g = 0; g < (PAIRED ? NG / 2 : NG); ++g) {
            double e0[VE], e1[VE];
            VT outv[VE];
#pragma unroll
            for (int v = 0; v < VE; ++v) e0[v] = e1[v] = 0.0;
            if constexpr (PAIRED) {
                outv[0] = VT(acc[2 * g][0]);
                outv[1] = VT(acc[2 * g + 1][0]);
                outv[2] = VT(acc[2 * g][1]);
                outv[3] = VT(acc[2 * g + 1][1]);
            } else {
                outv[0] = VT(acc[g][0]);
                outv[1] = VT(acc[g][1]);
            }
            const int col0 = PAIRED ? 16 * g + 4 * fc : 8 * g + 2 * fc;
            finish_row<VT, VE, CV>(a, i * 8 + fr, col0 / VE, outv, e0, e1);
            if (ndots) {
#pragma unroll
                for (int o = 4; o < 32; o <<= 1)
#pragma unroll
                    for (int v = 0; v < VE; ++v) {
                        e0[v] += __shfl_xor_sync(0xffffffffu, e0[v], o);
                        if (ndots == 2) e1[v] += __shfl_xor_sync(0xffffffffu, e1[v], o);
                    }
                if (fr == 0)
#pragma unroll
                    for (int v = 0; v < VE; ++v) {
                        dsm[warp][0][col0 + v] += e0[v];
                        dsm[warp][1][col0 + v] += e1[v];
                    }
            }
        }
    }
    if (ndots) {
        __syncthreads();
        double* mine = a.partials + size_t(blockIdx.x) * ndots * W;
        for (int idx = threadIdx.x; idx < ndots * W; idx += blockDim.x) {
            const int d = idx / W, col = idx - d * W;
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < kDmmaWarps; ++w) s += dsm[w][d][col];
            mine[idx] = s;
        }
        finish_partials(a, ndots);
    }
}

}  // namespace rsatb_b200
