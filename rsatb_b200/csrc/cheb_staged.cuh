// Shared-memory staged variant of the fused Chebyshev step.
//
// Same arithmetic and epilogue as cheb_step_kernel, but every operand of
// the inner loop arrives through a per-warp cp.async pipeline of STAGES
// blocks: for block k of a block row the X_j rows (each lane copies its own
// V values of every row, so it reads back only what it copied) and the
// b x b block of A (copied cooperatively by the lanes that share the block
// row, read back with uniform shared-memory loads).  Blocks k+1 ..
// k+STAGES-1 are in flight while block k is multiplied, which hides the
// DRAM latency of the streamed A values and the L2 latency of the gathered
// X rows without holding prefetched values in registers.
//
// Thread mapping: L = W / V lanes cover one block row.  L <= 32: a warp holds
// 32 / L block rows (sub-groups of L lanes).  L > 32: the block row is split
// into n_chunks = L / 32 column chunks, one warp each.  Work items (block
// row, chunk) are spread grid-stride over the sub-groups; CTA sizes keep
// every thread on a fixed column group, so the per-thread FP64 dot partials
// stay valid across items.
#pragma once

#include "cheb_kernels.cuh"

namespace rsatb_b200 {

template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    if constexpr (BYTES == 16) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(BYTES)
                     : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Largest of 16/8/4 dividing n bytes.
template <int NBYTES>
struct CopyChunk {
    static constexpr int value = (NBYTES % 16 == 0) ? 16 : ((NBYTES % 8 == 0) ? 8 : 4);
};

// Copies NBYTES (multiple of 4) with cp.async chunks, one thread.
template <int NBYTES>
__device__ __forceinline__ void cp_async_span(void* smem, const void* gmem) {
    constexpr int C = CopyChunk<NBYTES>::value;
#pragma unroll
    for (int o = 0; o < NBYTES; o += C)
        cp_async<C>(static_cast<char*>(smem) + o, static_cast<const char*>(gmem) + o);
}

// Shared-memory vector loads (same shape rules as load_vals).
template <typename T, int N>
__device__ __forceinline__ void lds_vals(const T* p, T (&o)[N]) {
    if constexpr (sizeof(T) == 8 && N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N / 2; ++i) {
            const double2 t = reinterpret_cast<const double2*>(p)[i];
            o[2 * i] = t.x;
            o[2 * i + 1] = t.y;
        }
    } else if constexpr (sizeof(T) == 4 && N % 4 == 0) {
#pragma unroll
        for (int i = 0; i < N / 4; ++i) {
            const float4 t = reinterpret_cast<const float4*>(p)[i];
            o[4 * i] = t.x;
            o[4 * i + 1] = t.y;
            o[4 * i + 2] = t.z;
            o[4 * i + 3] = t.w;
        }
    } else if constexpr (sizeof(T) == 4 && N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N / 2; ++i) {
            const float2 t = reinterpret_cast<const float2*>(p)[i];
            o[2 * i] = t.x;
            o[2 * i + 1] = t.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) o[i] = p[i];
    }
}

// Shared bytes one warp uses: STAGES x (X rows + one A block per sub-group),
// rounded to 16 bytes.
template <typename VT, typename MT, int B, int V, bool CM, int STAGES>
__host__ __device__ constexpr int staged_warp_bytes(int sg_per_warp) {
    return ((STAGES * (B * 32 * V * int(sizeof(VT)) +
                       sg_per_warp * B * B * (CM ? 2 : 1) * int(sizeof(MT))) +
             15) / 16) * 16;
}

// CTA reduction for the staged mapping, then the last-CTA reduction.
template <int V>
__device__ __forceinline__ void reduce_dots_staged(const StepArgs& a, int Lp, int n_chunks,
                                                   const double (&d0)[V], const double (&d1)[V]) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* red = reinterpret_cast<double*>(smem_raw);  // reuses the staging area
    __syncthreads();
    const int ndots = (a.dot_mode == DOT_DOUBLING) ? 2 : 1;
    const int nt = blockDim.x;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        red[threadIdx.x * V + v] = d0[v];
        if (ndots == 2) red[(nt + threadIdx.x) * V + v] = d1[v];
    }
    __syncthreads();
    const int W = a.W;
    const int spw = 32 / Lp;
    double* mine = a.partials + size_t(blockIdx.x) * ndots * W;
    for (int idx = threadIdx.x; idx < ndots * W; idx += nt) {
        const int d = idx / W, w = idx - d * W;
        const int g = w / V, v = w - g * V;
        const int ch = g / Lp, li = g - ch * Lp;
        double s = 0.0;
        if (n_chunks == 1) {
            for (int t = li; t < nt; t += Lp) s += red[(d * nt + t) * V + v];
        } else {
            for (int t = 0; t < nt; ++t) {
                const int lane = t & 31;
                if (lane % Lp != li) continue;
                if ((((t >> 5) * spw + lane / Lp) % n_chunks) != ch) continue;
                s += red[(d * nt + t) * V + v];
            }
        }
        mine[idx] = s;
    }
    finish_partials(a, ndots);
}

template <typename VT, typename MT, int B, int V, bool CM, bool CV, int STAGES>
__global__ void __launch_bounds__(256) cheb_step_staged(StepArgs a, int Lp, int n_chunks) {
    static_assert(!CV || V % 2 == 0, "complex panels need (re, im) pairs per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int RW = B * (CM ? 2 : 1);       // values per block row of A
    constexpr int BBV = B * RW;                 // values per block
    constexpr int XS = B * 32 * V;              // X values per stage per warp
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int spw = 32 / Lp;
    const int sg_local = lane / Lp, lane_in = lane - sg_local * Lp;
    unsigned char* wbase =
        smem_raw + size_t(warp) * staged_warp_bytes<VT, MT, B, V, CM, STAGES>(spw);
    VT* xs = reinterpret_cast<VT*>(wbase);
    MT* as = reinterpret_cast<MT*>(wbase + STAGES * XS * sizeof(VT));
    const unsigned gmask =
        (Lp == 32) ? 0xffffffffu : (((1u << Lp) - 1u) << (sg_local * Lp));

    const int W = a.W;
    const int64_t total_items = a.n_block_rows * n_chunks;
    const int64_t total_sg = int64_t(gridDim.x) * (blockDim.x >> 5) * spw;
    const int64_t sg0 = (int64_t(blockIdx.x) * (blockDim.x >> 5) + warp) * spw + sg_local;
    const int ch = int(sg0 % n_chunks);
    const int g = ch * Lp + lane_in;
    const MT* __restrict__ vals = static_cast<const MT*>(a.vals);
    const VT* __restrict__ in = static_cast<const VT*>(a.in);

    double d0[V], d1[V];
#pragma unroll
    for (int v = 0; v < V; ++v) d0[v] = d1[v] = 0.0;

    for (int64_t item = sg0; item < total_items; item += total_sg) {
        const int64_t i = item / n_chunks;
        const int k0 = __ldg(a.row_ptr + i), k1 = __ldg(a.row_ptr + i + 1);
        auto issue = [&](int k, int stage) {
            const int64_t j = __ldg(a.col_ind + k);
            VT* xdst = xs + stage * XS + lane * V;
#pragma unroll
            for (int c = 0; c < B; ++c)
                cp_async_span<V * int(sizeof(VT))>(xdst + c * 32 * V,
                                                   in + (j * B + c) * W + int64_t(g) * V);
            constexpr int ABYTES = BBV * int(sizeof(MT));
            constexpr int C = CopyChunk<ABYTES>::value;
            constexpr int NCH = ABYTES / C;
            const char* asrc = reinterpret_cast<const char*>(vals + int64_t(k) * BBV);
            char* adst = reinterpret_cast<char*>(as + (stage * spw + sg_local) * BBV);
            for (int q = lane_in; q < NCH; q += Lp) cp_async<C>(adst + q * C, asrc + q * C);
        };
#pragma unroll
        for (int s = 0; s < STAGES - 1; ++s) {
            if (k0 + s < k1) issue(k0 + s, s);
            cp_async_commit();
        }
        VT acc[B][V];
#pragma unroll
        for (int r = 0; r < B; ++r)
#pragma unroll
            for (int v = 0; v < V; ++v) acc[r][v] = VT(0);
        for (int k = k0; k < k1; ++k) {
            const int kk = k - k0;
            if (k + STAGES - 1 < k1) issue(k + STAGES - 1, (kk + STAGES - 1) % STAGES);
            cp_async_commit();
            VT xb[B][V];
            cp_async_wait<STAGES - 1>();
            __syncwarp(gmask);
            const int stage = kk % STAGES;
            const VT* xsrc = xs + stage * XS + lane * V;
#pragma unroll
            for (int c = 0; c < B; ++c) lds_vals<VT, V>(xsrc + c * 32 * V, xb[c]);
            const MT* blk = as + (stage * spw + sg_local) * BBV;
#pragma unroll
            for (int r = 0; r < B; ++r) {
                MT arow[RW];
                lds_vals<MT, RW>(blk + r * RW, arow);
#pragma unroll
                for (int c = 0; c < B; ++c) {
                    if constexpr (CM) {
                        const VT ar = VT(arow[2 * c]);
                        const VT ai = VT(arow[2 * c + 1]);
#pragma unroll
                        for (int v = 0; v < V; v += 2) {
                            acc[r][v] = fma(ar, xb[c][v], acc[r][v]);
                            acc[r][v] = fma(-ai, xb[c][v + 1], acc[r][v]);
                            acc[r][v + 1] = fma(ar, xb[c][v + 1], acc[r][v + 1]);
                            acc[r][v + 1] = fma(ai, xb[c][v], acc[r][v + 1]);
                        }
                    } else {
                        const VT av = VT(arow[c]);
#pragma unroll
                        for (int v = 0; v < V; ++v) acc[r][v] = fma(av, xb[c][v], acc[r][v]);
                    }
                }
            }
            __syncwarp(gmask);  // this stage is refilled STAGES-1 iterations later
        }
        cp_async_wait<0>();
#pragma unroll
        for (int r = 0; r < B; ++r) finish_row<VT, V, CV>(a, i * B + r, g, acc[r], d0, d1);
    }
    if (a.dot_mode != DOT_NONE) reduce_dots_staged<V>(a, Lp, n_chunks, d0, d1);
}

}  // namespace rsatb_b200
