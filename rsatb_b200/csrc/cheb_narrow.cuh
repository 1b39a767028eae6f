// Narrow-panel fused Chebyshev step: real 8x8 blocks, panels of 4 to 16
// real values per row, FP32 or FP64.
//
// At narrow panels the step is bound by streaming A (256 or 512 bytes per
// block against 8 W values of gathered X), so what matters is how many L1
// wavefronts a block costs.  The register and staged kernels let every
// block row (1 to 4 lanes) fetch its own blocks: each warp-wide load then
// touches 8 to 32 different blocks and a block costs about 22 wavefronts.
// Here a warp walks S = 32 / G block rows in lock step (G = W / V lanes per
// block row, V panel values per lane) and, at every step, the whole warp
// copies the step's S blocks of A and S gathered X_j blocks (8 rows of W
// values, contiguous in the row-major panel) into a shared-memory stage
// with 16-byte cp.async chunks: consecutive lanes take consecutive chunks
// of one block, so every copy instruction reads whole 128-byte lines.  The
// block and column indices travel from the block row's lane by shuffles.
// NS stages are in flight; a lane then multiplies its 8 x V register tile
// from conflict-free shared-memory reads (slots padded by 16 bytes).  The
// epilogue is finish_row; the per-thread FP64 dot partials live in shared
// memory and are reduced in a fixed order (deterministic).
#pragma once

#include "cheb_kernels.cuh"
#include "cheb_staged.cuh"

namespace rsatb_b200 {

constexpr int kNarrowWarps = 4;

template <typename VT, int W>
struct NarrowShape {
    static constexpr int V = W < 4 ? W : 4;                // panel values per lane
    static constexpr int G = W / V;                        // lanes per block row
    static constexpr int S = 32 / G;                       // block rows per warp
    static constexpr int ABYTES = 64 * int(sizeof(VT));    // one 8x8 block
    static constexpr int XBYTES = 8 * W * int(sizeof(VT)); // X_j: 8 rows of W values
    static constexpr int ACH = ABYTES / 16, XCH = XBYTES / 16, CH = ACH + XCH;
    static constexpr int ASLOT = ABYTES + 16, XSLOT = XBYTES + 16;
    static constexpr int XBASE = S * ASLOT;
    static constexpr int STAGE = S * (ASLOT + XSLOT);
    static constexpr int ITER = S * CH / 32;               // copy instructions per lane per step
    static_assert(W % V == 0 && 32 % G == 0 && XBYTES % 16 == 0, "narrow shape");
    static_assert((S * CH) % 32 == 0, "whole copy rounds");
};

// Per CTA: the warps' rings, then per warp and stage the (block, column
// block) pairs of the step's S block rows.
template <typename VT, int W, int NS>
constexpr size_t narrow_smem_bytes() {
    using Sh = NarrowShape<VT, W>;
    return size_t(kNarrowWarps) * NS * (Sh::STAGE + Sh::S * 8);
}

template <typename VT, int W, bool CV, int NS>
__global__ void __launch_bounds__(kNarrowWarps * 32) cheb_step_narrow(StepArgs a) {
    using Sh = NarrowShape<VT, W>;
    constexpr int V = Sh::V, G = Sh::G, S = Sh::S;
    static_assert(!CV || V % 2 == 0, "complex panels need (re, im) pairs per lane");
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* ring = smem + size_t(warp) * NS * Sh::STAGE;
    int2* table = reinterpret_cast<int2*>(smem + size_t(kNarrowWarps) * NS * Sh::STAGE) +
                  size_t(warp) * NS * S;
    const int u = lane / G, h = lane % G;  // block row in the group, column group
    const int64_t nbr = a.n_block_rows;
    const int64_t n_groups = (nbr + S - 1) / S;
    const int64_t nw = int64_t(gridDim.x) * kNarrowWarps;
    const int64_t wg = int64_t(blockIdx.x) * kNarrowWarps + warp;
    const char* __restrict__ vals = static_cast<const char*>(a.vals);
    const char* __restrict__ in = static_cast<const char*>(a.in);

    // Producer (NS - 1 steps ahead of the consumer): this lane's block row
    // u of the producer group; pj = column block of the step to issue,
    // loaded one step early.
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
        pj = pnk > 0 ? __ldg(a.col_ind + pk0) : 0;
    };
    auto p_issue = [&](int st) {
        unsigned char* stage = ring + st * Sh::STAGE;
        int2* tab = table + st * S;
        if (h == 0) tab[u] = make_int2(pt < pnk ? pk0 + pt : -1, pj);
        if (pt + 1 < pnk) pj = __ldg(a.col_ind + pk0 + pt + 1);
        __syncwarp();
#pragma unroll 4
        for (int it = 0; it < Sh::ITER; ++it) {
            const int id = it * 32 + lane;
            const int su = id / Sh::CH, ch = id - su * Sh::CH;
            const int2 kj = tab[su];
            if (kj.x >= 0) {
                if (ch < Sh::ACH)
                    cp_async<16>(stage + su * Sh::ASLOT + ch * 16,
                                 vals + int64_t(kj.x) * Sh::ABYTES + ch * 16);
                else
                    cp_async<16>(stage + Sh::XBASE + su * Sh::XSLOT + (ch - Sh::ACH) * 16,
                                 in + int64_t(kj.y) * Sh::XBYTES + (ch - Sh::ACH) * 16);
            }
        }
        if (++pt == psteps) {
            pgrp += nw;
            pt = 0;
            p_load();
        }
    };

    // Consumer.
    int64_t cgrp = wg;
    int ct = 0, csteps = 1, cnk = 0;
    auto c_load = [&]() {
        const int64_t i = cgrp * S + u;
        cnk = 0;
        if (cgrp < n_groups && i < nbr) cnk = __ldg(a.row_ptr + i + 1) - __ldg(a.row_ptr + i);
        csteps = max(1, int(__reduce_max_sync(0xffffffffu, unsigned(cnk))));
    };

    p_load();
    c_load();
#pragma unroll
    for (int st = 0; st < NS - 1; ++st) {
        if (pgrp < n_groups) p_issue(st);
        cp_async_commit();
    }

    VT acc[8][V];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int v = 0; v < V; ++v) acc[r][v] = VT(0);
    double d0[V], d1[V];
#pragma unroll
    for (int v = 0; v < V; ++v) d0[v] = d1[v] = 0.0;

    int st = 0;  // stage of the current step
    for (; cgrp < n_groups; st = (st + 1 == NS) ? 0 : st + 1) {
        // Refill the stage read one step ago with the step NS - 1 ahead.
        if (pgrp < n_groups) p_issue(st == 0 ? NS - 1 : st - 1);
        cp_async_commit();
        cp_async_wait<NS - 1>();
        __syncwarp();
        if (ct < cnk) {
            const unsigned char* stage = ring + st * Sh::STAGE;
            const VT* As = reinterpret_cast<const VT*>(stage + u * Sh::ASLOT);
            const VT* Xs = reinterpret_cast<const VT*>(stage + Sh::XBASE + u * Sh::XSLOT);
            VT xr[8][V];
#pragma unroll
            for (int c = 0; c < 8; ++c) lds_vals<VT, V>(Xs + c * W + h * V, xr[c]);
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                VT ar[8];
                lds_vals<VT, 8>(As + r * 8, ar);
#pragma unroll
                for (int c = 0; c < 8; ++c) fma_row<VT, V>(acc[r], ar[c], xr[c]);
            }
        }
        __syncwarp();  // this stage is refilled at the next step
        if (++ct == csteps) {
            const int64_t i = cgrp * S + u;
            if (i < nbr) {
#pragma unroll
                for (int r = 0; r < 8; ++r) finish_row<VT, V, CV>(a, i * 8 + r, h, acc[r], d0, d1);
            }
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int v = 0; v < V; ++v) acc[r][v] = VT(0);
            cgrp += nw;
            ct = 0;
            c_load();
        }
    }
    cp_async_wait<0>();
    if (a.dot_mode != DOT_NONE) {
        __syncthreads();  // the rings are free: reduce_dots reuses shared memory
        reduce_dots<V>(a, G, d0, d1);
    }
}

}  // namespace rsatb_b200
