// Fused Chebyshev step fed by bulk copies: FP32 panels, real 8x8 blocks.
//
// The register kernel (cheb_step_kernel) reads each 8x8 block of A with
// 128-bit loads that every lane of a block row issues for the same address;
// the L1 serves such a load in four quarter-warp passes, so at V = 4 values
// per lane the A reads cost twice the L1 wavefronts of the X gathers.  Here
//
//  * each warp owns S = 32 / G block rows (G = W / 8 lanes per block row,
//    8 panel values per lane: columns 4g..4g+3 and W/2+4g..W/2+4g+3) and
//    walks their blocks in lock step;
//  * the A blocks of the next NS steps are brought into a per-warp
//    shared-memory ring by 1-D bulk copies (cp.async.bulk, completion on one
//    mbarrier per stage) and read back as 32-bit broadcasts (slots padded to
//    spread the banks); at 8 columns per lane every A value feeds 8 FMAs;
//  * the gathered X_j rows (8 rows x W values, contiguous in the row-major
//    panel) are read with L1-cached 128-bit global loads (XG), so block rows
//    that share a column block on one SM share its L1 lines; the variant
//    XG = false brings X_j through the ring as well (measured slower: every
//    X byte then crosses shared memory twice);
//  * the FMAs are issued as packed pairs (fma.rn.f32x2), half the issue
//    slots of scalar FMAs at the same per-output operation order;
//  * DUP: after its stage lands, the warp rewrites its A blocks in shared
//    memory transposed and with every value twice, [c][r] as (a, a) pairs,
//    so one 128-bit load gives the packed operands {a_rc, a_rc} and
//    {a_r+1,c, a_r+1,c} of two rows: a quarter of the 32-bit loads of the
//    row-major slot, and no register moves to build the broadcast pairs
//    (the arithmetic, and so every result bit, is the same).
//
// Every mbarrier wait is bounded by the global timer; a wait that gives up
// poisons the dots with NaN, sets *fault and leaves the loop.  The epilogue
// (rescale, recurrence, store, FP64 dots) is finish_row; the per-thread dot
// partials live in shared memory and are reduced in a fixed order, then by
// finish_partials (deterministic).
#pragma once

#include "cheb_kernels.cuh"
#include "umma.cuh"

namespace rsatb_b200 {

constexpr int kBulkWarps = 4;
constexpr uint64_t kBulkWaitNs = 2000000000ull;  // 2 s per wait

// Per-warp ring layout.  XG: X rows are read straight from global memory
// (L1-cached) and only the A blocks travel through the ring.
template <int W, bool XG>
struct BulkShape {
    static constexpr int G = W / 8;            // lanes per block row
    static constexpr int S = 32 / G;           // block rows per warp
    static constexpr int ASLOT = 272;          // 8x8 FP32 block + 16 B (bank spread)
    static constexpr int XSLOT = 32 * W + 16;  // X_j: 8 rows x W values + 16 B
    static constexpr int STAGE = S * ASLOT + (XG ? 0 : S * XSLOT);
    static constexpr int XBASE = S * ASLOT;
    static constexpr unsigned BYTES = 256u + (XG ? 0u : unsigned(32 * W));  // per block row
    // DUP slot (floats): 8 columns c of 20 (8 pairs + 4 pad: rows 16-byte
    // aligned, the pair stores of a warp spread over the banks), + 4 pad so
    // the S slots of a warp start in different banks.
    static constexpr int DROW = 20;
    static constexpr int DSLOT = 8 * DROW + 4;
};

// Shared memory of one CTA: the warps' rings, the per-thread FP64 dot
// partials [threads][16] (d0 of both column groups, then d1), then the
// warps' DUP slots.
template <int W, bool XG, int NS>
constexpr size_t bulk_dup_offset() {
    return size_t(kBulkWarps) * NS * BulkShape<W, XG>::STAGE +
           size_t(kBulkWarps) * 32 * 16 * sizeof(double);
}
template <int W, bool XG, int NS>
constexpr size_t bulk_smem_bytes() {
    return bulk_dup_offset<W, XG, NS>() +
           size_t(kBulkWarps) * BulkShape<W, XG>::S * BulkShape<W, XG>::DSLOT * sizeof(float);
}

// (d0, d1) += (a0, a1) * (b0, b1) as one fma.rn.f32x2 (a0 = a1 for a
// broadcast A value held as a register pair).
__device__ __forceinline__ void fma2p(float& d0, float& d1, float a0, float a1, float b0,
                                      float b1) {
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rd, {%0, %1};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rd;\n\t"
        "mov.b64 {%0, %1}, rd;\n\t}"
        : "+f"(d0), "+f"(d1)
        : "f"(a0), "f"(a1), "f"(b0), "f"(b1));
}

// MINB: resident CTAs per SM the register budget is sized for; DUP: A read
// from the transposed, duplicated slot (see above).
template <int W, bool CV, int NS, bool XG, int MINB, bool DUP>
__global__ void __launch_bounds__(kBulkWarps * 32, MINB) cheb_step_bulk(StepArgs a) {
    using Sh = BulkShape<W, XG>;
    constexpr int G = Sh::G, S = Sh::S;
    static_assert(W % 8 == 0 && 32 % (W / 8) == 0, "8 values per lane; G must divide 32");
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bars[kBulkWarps][NS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* ring = smem + size_t(warp) * NS * Sh::STAGE;
    double* dsm = reinterpret_cast<double*>(smem + size_t(kBulkWarps) * NS * Sh::STAGE) +
                  size_t(threadIdx.x) * 16;
    float* dup = reinterpret_cast<float*>(smem + bulk_dup_offset<W, XG, NS>()) +
                 size_t(warp) * S * Sh::DSLOT;
    const int s = lane / G, g = lane % G;
    const int u = lane % S;  // the block row this lane copies (lanes < S issue)
    const int64_t nbr = a.n_block_rows;
    const int64_t n_groups = (nbr + S - 1) / S;
    const int64_t nw = int64_t(gridDim.x) * kBulkWarps;
    const int64_t wg = int64_t(blockIdx.x) * kBulkWarps + warp;
    const float* __restrict__ vals = static_cast<const float*>(a.vals);
    const float* __restrict__ in = static_cast<const float*>(a.in);

#pragma unroll
    for (int v = 0; v < 16; ++v) dsm[v] = 0.0;
    if (lane == 0) {
        for (int st = 0; st < NS; ++st) umma::mbar_init(&bars[warp][st], 1);
        umma::fence_mbarrier_init();
    }
    __syncwarp();
    if (a.wait_check) {
        // Arm stage 0 for 16 bytes that no copy delivers: the bounded wait
        // runs out, records the fault and the kernel leaves (no copy issued).
        if (lane == 0) umma::mbar_arrive_expect_tx(&bars[warp][0], 16u);
        __syncwarp();
        const bool got = umma::mbar_wait(&bars[warp][0], 0u, 5000000ull);
        if (!__all_sync(0xffffffffu, got) && lane == 0 && a.fault) atomicOr(a.fault, 1u);
        return;
    }

    // Producer: the item sequence (group, step) NS items ahead of the
    // consumer; pj holds the column block of the current producer item.
    int64_t pgrp = wg;
    int pt = 0, psteps = 1, pk0 = 0, pnk = 0, pj = 0;
    auto p_load = [&]() {
        const int64_t i = pgrp * S + u;
        pk0 = 0;
        pnk = 0;
        if (pgrp < n_groups && i < nbr) {
            pk0 = __ldg(a.row_ptr + i);
            pnk = __ldg(a.row_ptr + i + 1) - pk0;
        }
        psteps = max(1, int(__reduce_max_sync(0xffffffffu, unsigned(pnk))));
        if constexpr (!XG) pj = (lane < S && pnk > 0) ? __ldg(a.col_ind + pk0) : 0;
    };
    auto p_issue = [&](int st) {
        unsigned char* stage = ring + st * Sh::STAGE;
        const bool has = lane < S && pt < pnk;
        const unsigned total = __reduce_add_sync(0xffffffffu, has ? Sh::BYTES : 0u);
        if (lane == 0) umma::mbar_arrive_expect_tx(&bars[warp][st], total);
        __syncwarp();
        if (has) {
            umma::fence_proxy_async_smem();
            umma::bulk_load(stage + u * Sh::ASLOT, vals + int64_t(pk0 + pt) * 64, 256u,
                            &bars[warp][st]);
            if constexpr (!XG)
                umma::bulk_load(stage + Sh::XBASE + u * Sh::XSLOT, in + int64_t(pj) * 8 * W,
                                unsigned(32 * W), &bars[warp][st]);
        }
        if (++pt == psteps) {
            pgrp += nw;
            pt = 0;
            p_load();
        } else if (!XG && lane < S && pt < pnk) {
            pj = __ldg(a.col_ind + pk0 + pt);
        }
    };

    // Consumer; cj is the column block of the current item (XG).
    int64_t cgrp = wg;
    int ct = 0, csteps = 1, cnk = 0, ck0 = 0, cj = 0;
    auto c_load = [&]() {
        const int64_t i = cgrp * S + s;
        cnk = 0;
        if (cgrp < n_groups && i < nbr) {
            ck0 = __ldg(a.row_ptr + i);
            cnk = __ldg(a.row_ptr + i + 1) - ck0;
        }
        csteps = max(1, int(__reduce_max_sync(0xffffffffu, unsigned(cnk))));
        if constexpr (XG) cj = cnk > 0 ? __ldg(a.col_ind + ck0) : 0;
    };

    p_load();
    c_load();
    for (int st = 0; st < NS; ++st)
        if (pgrp < n_groups) p_issue(st);

    float acc[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[r][v] = 0.f;
    bool failed = false;

    int st = 0;        // stage of the current item
    uint32_t par = 0;  // its mbarrier phase parity
    for (; cgrp < n_groups; st = (st + 1 == NS) ? 0 : st + 1, par ^= (st == 0)) {
        const bool live = ct < cnk;
        const float* xb = in + int64_t(cj) * 8 * W + 4 * g;
        if constexpr (XG) {
            if (live && ct + 1 < cnk) cj = __ldg(a.col_ind + ck0 + ct + 1);
        }
        const bool got = umma::mbar_wait(&bars[warp][st], par, kBulkWaitNs);
        if (!__all_sync(0xffffffffu, got)) {
            failed = true;
            break;
        }
        if constexpr (DUP) {
            // Rewrite the stage's S blocks as [c][r] (a, a) pairs (slots of
            // rows that have no block here hold stale values nobody reads).
            const float* sa = reinterpret_cast<const float*>(ring + st * Sh::STAGE);
#pragma unroll
            for (int u = 0; u < 2 * S; ++u) {
                const int idx = lane + 32 * u;
                const int b = idx >> 6, e = idx & 63;
                const float v = sa[b * (Sh::ASLOT / 4) + e];
                *reinterpret_cast<float2*>(dup + b * Sh::DSLOT + (e & 7) * Sh::DROW + 2 * (e >> 3)) =
                    make_float2(v, v);
            }
            __syncwarp();
        }
        if (live) {
            const unsigned char* stage = ring + st * Sh::STAGE;
            const float* As = reinterpret_cast<const float*>(stage + s * Sh::ASLOT);
            const float* Xs = reinterpret_cast<const float*>(stage + Sh::XBASE + s * Sh::XSLOT);
            const float* Ds = dup + s * Sh::DSLOT;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                float4 x0, x1;
                if constexpr (XG) {
                    x0 = __ldg(reinterpret_cast<const float4*>(xb + c * W));
                    x1 = __ldg(reinterpret_cast<const float4*>(xb + c * W + W / 2));
                } else {
                    x0 = *reinterpret_cast<const float4*>(Xs + c * W + 4 * g);
                    x1 = *reinterpret_cast<const float4*>(Xs + c * W + W / 2 + 4 * g);
                }
                if constexpr (DUP) {
#pragma unroll
                    for (int rp = 0; rp < 4; ++rp) {
                        const float4 aa =
                            *reinterpret_cast<const float4*>(Ds + c * Sh::DROW + 4 * rp);
                        float* u0 = acc[2 * rp];
                        float* u1 = acc[2 * rp + 1];
                        fma2p(u0[0], u0[1], aa.x, aa.y, x0.x, x0.y);
                        fma2p(u0[2], u0[3], aa.x, aa.y, x0.z, x0.w);
                        fma2p(u0[4], u0[5], aa.x, aa.y, x1.x, x1.y);
                        fma2p(u0[6], u0[7], aa.x, aa.y, x1.z, x1.w);
                        fma2p(u1[0], u1[1], aa.z, aa.w, x0.x, x0.y);
                        fma2p(u1[2], u1[3], aa.z, aa.w, x0.z, x0.w);
                        fma2p(u1[4], u1[5], aa.z, aa.w, x1.x, x1.y);
                        fma2p(u1[6], u1[7], aa.z, aa.w, x1.z, x1.w);
                    }
                } else {
#pragma unroll
                    for (int r = 0; r < 8; ++r) {
                        const float av = As[r * 8 + c];
                        fma2(acc[r][0], acc[r][1], av, x0.x, x0.y);
                        fma2(acc[r][2], acc[r][3], av, x0.z, x0.w);
                        fma2(acc[r][4], acc[r][5], av, x1.x, x1.y);
                        fma2(acc[r][6], acc[r][7], av, x1.z, x1.w);
                    }
                }
            }
        }
        __syncwarp();  // stage st is read: refill it with the item NS ahead
        if (pgrp < n_groups) p_issue(st);
        if (++ct == csteps) {
            const int64_t i = cgrp * S + s;
            if (i < nbr) {
                double e0[4] = {0, 0, 0, 0}, e1[4] = {0, 0, 0, 0};
                double f0[4] = {0, 0, 0, 0}, f1[4] = {0, 0, 0, 0};
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    const float lo[4] = {acc[r][0], acc[r][1], acc[r][2], acc[r][3]};
                    const float hi[4] = {acc[r][4], acc[r][5], acc[r][6], acc[r][7]};
                    finish_row<float, 4, CV>(a, i * 8 + r, g, lo, e0, e1);
                    finish_row<float, 4, CV>(a, i * 8 + r, g + G, hi, f0, f1);
                }
                if (a.dot_mode != DOT_NONE) {
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        dsm[v] += e0[v];
                        dsm[4 + v] += f0[v];
                        dsm[8 + v] += e1[v];
                        dsm[12 + v] += f1[v];
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int v = 0; v < 8; ++v) acc[r][v] = 0.f;
            cgrp += nw;
            ct = 0;
            c_load();
        }
    }
    if (failed) {
        // A bounded wait gave up: record it and poison this thread's dots.
        if (lane == 0 && a.fault) atomicOr(a.fault, 1u);
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
#pragma unroll
        for (int v = 0; v < 16; ++v) dsm[v] = nan;
    }

    if (a.dot_mode != DOT_NONE) {
        __syncthreads();
        const double* red = reinterpret_cast<const double*>(smem + size_t(kBulkWarps) * NS * Sh::STAGE);
        const int nt = blockDim.x;
        const int t = threadIdx.x;
        const int ndots = a.dot_mode == DOT_DOUBLING ? 2 : 1;
        double* mine = a.partials + size_t(blockIdx.x) * ndots * W;
        for (int idx = t; idx < ndots * W; idx += nt) {
            const int d = idx / W, w = idx - d * W;
            const int q4 = w >> 2, v = w & 3;
            const int half = q4 / G, gg = q4 - half * G;
            const int col = d * 8 + half * 4 + v;
            double sum = 0.0;
            for (int tt = gg; tt < nt; tt += G) sum += red[tt * 16 + col];
            mine[idx] = sum;
        }
        finish_partials(a, ndots);
    }
}

}  // namespace rsatb_b200
