// Narrow-panel variant of the fused Chebyshev step (W <= 16 values per row),
// where the SpMM is bound by streaming A from HBM.
//
// One warp per block row.  Lane l takes output row r = l / KL of the block
// and the block columns c = KC*q .. KC*q + KC-1 (q = l % KL, KL lanes per
// row, KC = B / KL): one warp instruction then loads a whole b x b block of
// A as contiguous KC-value pieces (fully coalesced), and each lane reads the
// KC rows X_j[c, 0..W) it needs.  Lanes accumulate partial sums over their
// columns c for all W panel values; after the block row, a butterfly over
// the KL lanes of a row completes the sums, and lane q finishes the values
// [q*V, q*V + V) (V = W / KL) with the usual epilogue.  UNROLL blocks are
// loaded before they are multiplied to keep several A blocks in flight.
#pragma once

#include "cheb_kernels.cuh"

namespace rsatb_b200 {

template <int V>
__device__ __forceinline__ void reduce_dots_lanes(const StepArgs& a, int KL, int B,
                                                  const double (&d0)[V], const double (&d1)[V]) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* red = reinterpret_cast<double*>(smem_raw);
    const int ndots = (a.dot_mode == DOT_DOUBLING) ? 2 : 1;
    const int nt = blockDim.x;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        red[threadIdx.x * V + v] = d0[v];
        if (ndots == 2) red[(nt + threadIdx.x) * V + v] = d1[v];
    }
    __syncthreads();
    const int W = a.W;
    double* mine = a.partials + size_t(blockIdx.x) * ndots * W;
    for (int idx = threadIdx.x; idx < ndots * W; idx += nt) {
        const int d = idx / W, w = idx - d * W;
        const int g = w / V, v = w - g * V;
        double s = 0.0;
        for (int t = 0; t < nt; ++t) {
            const int lane = t & 31;
            if (lane % KL != g || lane / KL >= B) continue;
            s += red[(d * nt + t) * V + v];
        }
        mine[idx] = s;
    }
    finish_partials(a, ndots);
}

// VT: panel/matrix real type; B: block size; KL: lanes per block row
// (power of two, KL*B <= 32); WW: panel width (compile time); CV: complex.
template <typename VT, int B, int KL, int WW, bool CV, int UNROLL>
__global__ void __launch_bounds__(256) cheb_step_rowsplit(StepArgs a) {
    constexpr int KC = (B + KL - 1) / KL;  // block columns per lane
    constexpr int V = WW / KL;             // epilogue values per lane
    static_assert(WW % KL == 0, "panel width must split over the row lanes");
    static_assert(!CV || V % 2 == 0, "complex values must stay in one lane");
    const int lane = threadIdx.x & 31;
    const int r = lane / KL, q = lane % KL;
    const bool active = r < B;
    const int rr = active ? r : 0;
    const VT* __restrict__ vals = static_cast<const VT*>(a.vals);
    const VT* __restrict__ in = static_cast<const VT*>(a.in);
    const int64_t warps_total = int64_t(gridDim.x) * (blockDim.x >> 5);
    const int64_t warp0 = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);

    double d0[V], d1[V];
#pragma unroll
    for (int v = 0; v < V; ++v) d0[v] = d1[v] = 0.0;

    for (int64_t i = warp0; i < a.n_block_rows; i += warps_total) {
        const int k0 = __ldg(a.row_ptr + i), k1 = __ldg(a.row_ptr + i + 1);
        VT acc[WW];
#pragma unroll
        for (int w = 0; w < WW; ++w) acc[w] = VT(0);
        for (int k = k0; k < k1; k += UNROLL) {
            VT av[UNROLL][KC];
            VT xv[UNROLL][KC][WW];
#pragma unroll
            for (int u = 0; u < UNROLL; ++u) {
                const bool ok = (k + u < k1);
                const int kk = ok ? k + u : k0;
                const int64_t j = __ldg(a.col_ind + kk);
                if constexpr (B % KC == 0) {
                    // The lane's KC columns are contiguous and aligned: one
                    // vector load (a warp covers the whole block).
                    VT t[KC];
                    load_vals<VT, KC>(vals + int64_t(kk) * B * B + rr * B + q * KC, t);
#pragma unroll
                    for (int e = 0; e < KC; ++e) av[u][e] = (ok && active) ? t[e] : VT(0);
                } else {
#pragma unroll
                    for (int e = 0; e < KC; ++e) {
                        const int c = q * KC + e;
                        const bool use = ok && active && c < B;
                        av[u][e] = use ? __ldg(vals + int64_t(kk) * B * B + rr * B + c) : VT(0);
                    }
                }
#pragma unroll
                for (int e = 0; e < KC; ++e) {
                    const int c = q * KC + e;
                    const int cc = c < B ? c : 0;
                    load_vals<VT, WW>(in + (j * B + cc) * WW, xv[u][e]);
                }
            }
#pragma unroll
            for (int u = 0; u < UNROLL; ++u)
#pragma unroll
                for (int e = 0; e < KC; ++e)
#pragma unroll
                    for (int w = 0; w < WW; ++w) acc[w] = fma(av[u][e], xv[u][e][w], acc[w]);
        }
        // Complete the row sums across the KL lanes of the row.
#pragma unroll
        for (int off = 1; off < KL; off <<= 1)
#pragma unroll
            for (int w = 0; w < WW; ++w) acc[w] += __shfl_xor_sync(0xffffffffu, acc[w], off);
        if (active) {
            VT mine[V];
#pragma unroll
            for (int v = 0; v < V; ++v) mine[v] = acc[q * V + v];
            finish_row<VT, V, CV>(a, i * B + r, q, mine, d0, d1);
        }
    }
    if (a.dot_mode != DOT_NONE) reduce_dots_lanes<V>(a, KL, B, d0, d1);
}

}  // namespace rsatb_b200
