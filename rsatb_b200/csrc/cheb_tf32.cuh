// Fused Chebyshev step on the tensor cores for FP32 panels: real 8x8
// blocks, W = 64, 128 or 256 real values per row, split-TF32 products
// (mma.sync m16n8k8 tf32, three per tile) with FP32 accumulation.
//
// Orientation.  A block row's output is computed transposed,
//
//     Y_i^T (W x 8) = sum_j X_j^T (W x 8) . A_ij^T (8 x 8),
//
// so the panel columns are the MMA's M side (tiles of 16) and each 8x8
// block is one dense k8 x n8 B operand: no fill-in.  The B fragment
// (k = lane % 4 (+4), n = lane / 4) is A_ij[lane / 4][lane % 4 (+4)], the
// block in its row-major storage: two coalesced 32-bit loads per lane.  The
// A fragment (m = lane / 4 (+8), k = lane % 4 (+4)) is X_j^T: row k of X_j
// at the panel column that MMA row m stands for.  That column is free to
// choose, as long as the C fragment's row m is stored to the same column:
// lane group g = lane / 4 takes the 16-byte chunks g, g + 8, ... of its half
// of each X_j row, and tile t uses the lane's columns 2t (m = g) and 2t + 1
// (m = g + 8).  Every lane then reads whole float4 chunks of rows
// q = lane % 4 and q + 4 (a warp-wide load is four full 128-byte lines),
// and the accumulator leaves it rows 2q and 2q + 1 of the block row at its
// own columns, in 4-column chunks: the layout finish_row expects with V = 4.
//
// Work split.  Two warps share a block row, each half of the panel
// columns, so a warp's per-block registers (its X_j fragments, P = 2 or 3
// blocks deep) stay small.  The X_j rows are
// read with L1-cached 128-bit loads (neighbouring block rows of one CTA
// share their gathered lines); the next blocks' loads are in flight while a
// block is multiplied.
//
// Split TF32 and accuracy.  Each FP32 operand x is split as
// hi = rna_tf32(x), lo = x - hi (exact in FP32); a block's product is
// lo_a hi_b + hi_a lo_b + hi_a hi_b (the lo lo term is below FP32
// rounding), accumulated by the tensor core into a fresh tile per block,
// which is then added to the row's FP32 accumulator with IEEE adds.  The
// tensor core's own accumulation truncates; keeping it to one block's 24
// products and summing the blocks in rounded FP32 keeps the SpMM at FP32
// accuracy over rows of many blocks.
//
// Epilogue: finish_row (rescale, recurrence, store, FP64 dots), then the
// FP64 dot partials of one block row are summed over the four lanes of a
// group by shuffles (they share their columns) and kept per lane, each lane
// one chunk in four; at the end the warps' partials pass through shared
// memory, the CTA sums its warps in a fixed order and finish_partials sums
// the CTAs (deterministic).  No wait in this kernel can hang: it has no
// barrier other than __syncthreads and warp-synchronous MMAs.
#pragma once

#include "cheb_kernels.cuh"

namespace rsatb_b200 {

constexpr int kTf32Warps = 8;  // 4 block rows x 2 column halves per CTA

__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
    hi = h;
    lo = __float_as_uint(x - __uint_as_float(h));
}

// d = a b (C = 0) and d += a b on one m16n8k8 tf32 tile.
__device__ __forceinline__ void mma_tf32_zero(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                              uint32_t b1) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, "
        "{%4, %5, %6, %7}, {%8, %9}, {%10, %10, %10, %10};"
        : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(0.f));
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, "
        "{%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int W>
struct Tf32Shape {
    static_assert(W == 64 || W == 128 || W == 256, "W = 64, 128 or 256");
    static constexpr int WH = W / 2;   // columns per warp
    static constexpr int T = WH / 16;  // m16 tiles per warp
    static constexpr int NCH = T / 2;  // float4 chunks per lane and X row
};

// One block's operands in registers: X_j rows q and q + 4 at the lane's
// chunks, and the lane's two values of A_ij.
template <int NCH>
struct Tf32Block {
    float4 f0[NCH], f1[NCH];
    float b0, b1;
};

// P: blocks in flight per warp (2 or 3 register buffers); MINB: resident
// CTAs per SM the register budget is sized for.
template <int W, bool CV, int P, int MINB>
__global__ void __launch_bounds__(kTf32Warps * 32, MINB) cheb_step_tf32(StepArgs a) {
    static_assert(P == 2 || P == 3, "two or three blocks in flight");
    using Sh = Tf32Shape<W>;
    constexpr int WH = Sh::WH, T = Sh::T, NCH = Sh::NCH;
    __shared__ double red[kTf32Warps][2][WH];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, q = lane & 3;
    const int slot = warp >> 1, half = warp & 1;
    const int cbase = half * (WH / 4) + g;  // the lane's first chunk in a row
    const int64_t nbr = a.n_block_rows;
    const float* __restrict__ vals = static_cast<const float*>(a.vals);
    const float* __restrict__ in = static_cast<const float*>(a.in);
    const int ndots = a.dot_mode == DOT_DOUBLING ? 2 : (a.dot_mode == DOT_PLAIN ? 1 : 0);

    auto load = [&](Tf32Block<NCH>& B, int k) {
        const int64_t j = __ldg(a.col_ind + k);
        const float* xr = in + j * 8 * W + 4 * cbase;
#pragma unroll
        for (int v = 0; v < NCH; ++v) {
            B.f0[v] = __ldg(reinterpret_cast<const float4*>(xr + q * W + 32 * v));
            B.f1[v] = __ldg(reinterpret_cast<const float4*>(xr + (q + 4) * W + 32 * v));
        }
        const float* ab = vals + int64_t(k) * 64 + g * 8 + q;
        B.b0 = __ldg(ab);
        B.b1 = __ldg(ab + 4);
    };
    auto multiply = [&](const Tf32Block<NCH>& B, float (&acc)[T][4]) {
        uint32_t bh0, bl0, bh1, bl1;
        split_tf32(B.b0, bh0, bl0);  // A_ij[g][q]
        split_tf32(B.b1, bh1, bl1);  // A_ij[g][q + 4]
#pragma unroll
        for (int v = 0; v < NCH; ++v) {
            const float e0[4] = {B.f0[v].x, B.f0[v].y, B.f0[v].z, B.f0[v].w};
            const float e1[4] = {B.f1[v].x, B.f1[v].y, B.f1[v].z, B.f1[v].w};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint32_t ah[4], al[4];
                split_tf32(e0[2 * h], ah[0], al[0]);      // m = g,     k = q
                split_tf32(e0[2 * h + 1], ah[1], al[1]);  // m = g + 8, k = q
                split_tf32(e1[2 * h], ah[2], al[2]);      // m = g,     k = q + 4
                split_tf32(e1[2 * h + 1], ah[3], al[3]);  // m = g + 8, k = q + 4
                float c[4];
                mma_tf32_zero(c, al, bh0, bh1);
                mma_tf32(c, ah, bl0, bl1);
                mma_tf32(c, ah, bh0, bh1);
                float* t = acc[2 * v + h];
                t[0] += c[0];
                t[1] += c[1];
                t[2] += c[2];
                t[3] += c[3];
            }
        }
    };

    double dsum[2][4];
#pragma unroll
    for (int e = 0; e < 4; ++e) dsum[0][e] = dsum[1][e] = 0.0;

    for (int64_t i = int64_t(blockIdx.x) * (kTf32Warps / 2) + slot; i < nbr;
         i += int64_t(gridDim.x) * (kTf32Warps / 2)) {
        const int k0 = __ldg(a.row_ptr + i), k1 = __ldg(a.row_ptr + i + 1);
        float acc[T][4];
#pragma unroll
        for (int t = 0; t < T; ++t) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.f;
        Tf32Block<NCH> B0, B1, B2;
        if (k0 < k1) load(B0, k0);
        if (k0 + 1 < k1) load(B1, k0 + 1);
        if constexpr (P == 3) {
            if (k0 + 2 < k1) load(B2, k0 + 2);
        }
        for (int k = k0; k < k1; k += P) {
            multiply(B0, acc);
            if (k + P < k1) load(B0, k + P);
            if (k + 1 < k1) {
                multiply(B1, acc);
                if (k + 1 + P < k1) load(B1, k + 1 + P);
            }
            if constexpr (P == 3) {
                if (k + 2 < k1) {
                    multiply(B2, acc);
                    if (k + 5 < k1) load(B2, k + 5);
                }
            }
        }
        // Epilogue: rows 2q, 2q + 1 of block row i, the lane's chunks.
#pragma unroll
        for (int v = 0; v < NCH; ++v) {
            double e0[4] = {0, 0, 0, 0}, e1[4] = {0, 0, 0, 0};
            const float r0[4] = {acc[2 * v][0], acc[2 * v][2], acc[2 * v + 1][0],
                                 acc[2 * v + 1][2]};
            const float r1[4] = {acc[2 * v][1], acc[2 * v][3], acc[2 * v + 1][1],
                                 acc[2 * v + 1][3]};
            finish_row<float, 4, CV>(a, i * 8 + 2 * q, cbase + 8 * v, r0, e0, e1);
            finish_row<float, 4, CV>(a, i * 8 + 2 * q + 1, cbase + 8 * v, r1, e0, e1);
            if (ndots) {
#pragma unroll
                for (int o = 1; o < 4; o <<= 1)
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        e0[e] += __shfl_xor_sync(0xffffffffu, e0[e], o);
                        if (ndots == 2) e1[e] += __shfl_xor_sync(0xffffffffu, e1[e], o);
                    }
                if (v == q)
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        dsum[0][e] += e0[e];
                        dsum[1][e] += e1[e];
                    }
            }
        }
    }
    if (ndots) {
        // Each column of the warp's half is held by exactly one lane (chunk
        // g + 8v by the lane with q = v); NCH <= 4 chunks per lane group.
        if (q < NCH)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int col = 4 * (g + 8 * q) + e;
                red[warp][0][col] = dsum[0][e];
                red[warp][1][col] = dsum[1][e];
            }
        __syncthreads();
        double* mine = a.partials + size_t(blockIdx.x) * ndots * W;
        for (int idx = threadIdx.x; idx < ndots * W; idx += blockDim.x) {
            const int d = idx / W, col = idx - d * W;
            const int hf = col / WH, c = col - hf * WH;
            double s = 0.0;
#pragma unroll
            for (int sl = 0; sl < kTf32Warps / 2; ++sl) s += red[2 * sl + hf][d][c];
            mine[idx] = s;
        }
        finish_partials(a, ndots);
    }
}

}  // namespace rsatb_b200
