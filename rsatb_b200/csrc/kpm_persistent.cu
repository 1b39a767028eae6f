// Persistent KPM moment recurrence for small scalar-block (CSR) operators.
//
// A small operator (graphene pz: 7,200 rows, 3 nonzeros per row, 8 complex
// columns) is latency-bound: each of the 256 steps of a 512-moment
// recurrence moves ~1 MB, well inside L2, and a launch per step plus the
// last-CTA dot reduction cost more than the arithmetic.  Here one
// cooperative launch runs mu_0 and every step of the recurrence
// (rsatb/calc/dos.hpp:156-171): psi_1 = Op~ psi_0, psi_s = 2 Op~ psi_{s-1}
// - psi_{s-2}, with the step epilogue of the other kernels (finish_row,
// panels read through L2 since they are written earlier in the same
// launch).  Consecutive steps are separated by a grid barrier (all CTAs are
// co-resident: cooperative launch); its wait is bounded by the global timer
// and a wait that runs out sets the context's fault word and ends the
// launch.  Each CTA writes its per-step FP64 dot partials to its own slot;
// a second kernel sums the slots over CTAs in a fixed order, so the dots
// are deterministic.
#include "cheb_kernels.cuh"
#include "umma.cuh"

#include <algorithm>
#include <cstdlib>

namespace rsatb_b200 {
namespace {

constexpr uint64_t kGridWaitNs = 2000000000ull;  // 2 s per barrier
constexpr int kPersistSkipped = 1000;             // not launched: take the graph path

struct PersistArgs {
    StepArgs base;     // matrix, W, imag, c, s_out, dot mode
    const void* psi;   // psi_0
    void* buf[3];      // rotating panels
    int n_steps;
    double* part;      // [(n_steps + 1)][gridDim.x][2][W]
    unsigned* bar;     // grid barrier counter, zero at launch
};

// Grid barrier number `gen` (1, 2, ...): false when the wait ran out.
__device__ bool grid_barrier(unsigned* bar, unsigned gen) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        const unsigned target = gen * gridDim.x;
        int ok = 1;
        const uint64_t t0 = umma::global_timer_ns();
        while (true) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
            if (v >= target) break;
            if (umma::global_timer_ns() - t0 > kGridWaitNs) {
                ok = 0;
                break;
            }
        }
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// This CTA's dot partials of one step: threads t = g, g + L, ... hold the
// columns g*V .. g*V + V - 1; summed in thread order into out[ndots][W].
template <int V>
__device__ void cta_partials(int W, int L, int ndots, const double (&d0)[V],
                             const double (&d1)[V], double* red, double* out) {
    const int nt = blockDim.x, t = threadIdx.x;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        red[t * V + v] = d0[v];
        red[(nt + t) * V + v] = d1[v];
    }
    __syncthreads();
    for (int idx = t; idx < 2 * W; idx += nt) {
        const int d = idx / W, w = idx - d * W;
        const int g = w / V, v = w - g * V;
        double s = 0.0;
        if (d < ndots)
            for (int tt = g; tt < nt; tt += L) s += red[(d * nt + tt) * V + v];
        out[idx] = s;
    }
    __syncthreads();
}

template <typename VT, int V, bool CV>
__global__ void __launch_bounds__(256) kpm_persistent_kernel(PersistArgs pa) {
    __shared__ double red[2 * 256 * V];
    const StepArgs& b = pa.base;
    const int W = b.W, L = W / V;
    const int g = threadIdx.x % L;  // blockDim.x is a multiple of L
    const int64_t total = b.n_block_rows * L;  // scalar rows x lanes per row
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t t0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const VT* __restrict__ vals = static_cast<const VT*>(b.vals);
    const size_t slot = size_t(gridDim.x) * 2 * W;  // one step's partials
    const int ndots = b.dot_mode == DOT_DOUBLING ? 2 : 1;

    // mu_0 = <psi|psi> per column.
    {
        double d0[V], d1[V];
#pragma unroll
        for (int v = 0; v < V; ++v) d0[v] = d1[v] = 0.0;
        for (int64_t t = t0; t < total; t += stride) {
            const int64_t off = (t / L) * W + int64_t(g) * V;
            VT xv[V];
            load_vals<VT, V, true>(static_cast<const VT*>(pa.psi) + off, xv);
            if constexpr (CV) {
#pragma unroll
                for (int v = 0; v < V; v += 2)
                    d0[v] += double(xv[v]) * double(xv[v]) + double(xv[v + 1]) * double(xv[v + 1]);
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) d0[v] += double(xv[v]) * double(xv[v]);
            }
        }
        cta_partials<V>(W, L, 1, d0, d1, red, pa.part + size_t(blockIdx.x) * 2 * W);
    }

    // When every thread owns one row of at most kCache nonzeros (the grid
    // covers all rows), its column indices and values stay in registers for
    // the whole recurrence.
    constexpr int kCache = 8;
    const bool one_row = total <= stride;
    int nk = -1;
    int64_t cj[kCache];
    VT cv[kCache];
    if (one_row && t0 < total) {
        const int64_t i = t0 / L;
        const int k0 = __ldg(b.row_ptr + i), k1 = __ldg(b.row_ptr + i + 1);
        if (k1 - k0 <= kCache) {
            nk = k1 - k0;
#pragma unroll
            for (int q = 0; q < kCache; ++q) {
                cj[q] = q < nk ? __ldg(b.col_ind + k0 + q) : 0;
                cv[q] = q < nk ? __ldg(vals + k0 + q) : VT(0);
            }
        }
    }

    const VT* prev = nullptr;
    const VT* cur = static_cast<const VT*>(pa.psi);
    int bi = 0;
    for (int s = 1; s <= pa.n_steps; ++s) {
        VT* out = static_cast<VT*>(pa.buf[bi]);
        bi = bi == 2 ? 0 : bi + 1;
        StepArgs a = b;
        a.in = cur;
        a.x = cur;
        a.p = s == 1 ? nullptr : prev;
        a.y = out;
        a.s2 = s == 1 ? 1.0 : 2.0;
        a.g_p = s == 1 ? 0.0 : -1.0;
        double d0[V], d1[V];
#pragma unroll
        for (int v = 0; v < V; ++v) d0[v] = d1[v] = 0.0;
        if (nk >= 0) {
            const int64_t i = t0 / L;
            VT acc[V];
#pragma unroll
            for (int v = 0; v < V; ++v) acc[v] = VT(0);
            VT xv[kCache][V];
#pragma unroll
            for (int q = 0; q < kCache; ++q)
                if (q < nk) load_vals<VT, V, true>(cur + cj[q] * W + int64_t(g) * V, xv[q]);
#pragma unroll
            for (int q = 0; q < kCache; ++q)
                if (q < nk) fma_row<VT, V>(acc, cv[q], xv[q]);
            finish_row<VT, V, CV, true>(a, i, g, acc, d0, d1);
        } else {
            for (int64_t t = t0; t < total; t += stride) {
                const int64_t i = t / L;
                VT acc[V];
#pragma unroll
                for (int v = 0; v < V; ++v) acc[v] = VT(0);
                const int k0 = __ldg(b.row_ptr + i), k1 = __ldg(b.row_ptr + i + 1);
                for (int k = k0; k < k1; ++k) {
                    const int64_t j = __ldg(b.col_ind + k);
                    const VT av = __ldg(vals + k);
                    VT xv[V];
                    load_vals<VT, V, true>(cur + j * W + int64_t(g) * V, xv);
                    fma_row<VT, V>(acc, av, xv);
                }
                finish_row<VT, V, CV, true>(a, i, g, acc, d0, d1);
            }
        }
        cta_partials<V>(W, L, ndots, d0, d1, red,
                        pa.part + size_t(s) * slot + size_t(blockIdx.x) * 2 * W);
        if (s < pa.n_steps && !grid_barrier(pa.bar, unsigned(s))) {
            if (threadIdx.x == 0 && b.fault) atomicOr(b.fault, 1u);
            return;
        }
        prev = cur;
        cur = out;
    }
}

// dots[s][d][w] = sum over CTAs (in CTA order) of part[s][cta][d][w].
__global__ void persistent_dots_kernel(int n_slots, int grid, int W, const double* part,
                                       double* dots) {
    const int64_t n = int64_t(n_slots) * 2 * W;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
         e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t s = e / (2 * W), dw = e - s * 2 * W;
        const double* p = part + s * int64_t(grid) * 2 * W + dw;
        double acc = 0.0;
        for (int c = 0; c < grid; ++c) acc += p[int64_t(c) * 2 * W];
        dots[e] = acc;
    }
}

template <typename VT, int V, bool CV>
int launch_persistent(rsatb_context* ctx, PersistArgs pa, int64_t n_rows, double* dots,
                      size_t part_capacity) {
    auto kernel = kpm_persistent_kernel<VT, V, CV>;
    // The CTA size is a multiple of the L lanes of a row (W = 6: L = 3, 255
    // threads), so a thread's column group is threadIdx.x % L in every CTA
    // and at every grid stride, as the kernel and cta_partials assume.
    const int L = pa.base.W / V;
    if (L > 256) return kPersistSkipped;
    const int threads = 256 - 256 % L;
    int per_sm = 0;
    RSATB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0));
    if (per_sm < 1) return kPersistSkipped;
    int64_t grid = int64_t(ctx->sm_count) * per_sm;
    const int64_t need = (n_rows * L + threads - 1) / threads;
    if (need < grid) grid = need;
    // RSATB_PERSIST_CTAS caps the CTA count (fewer CTAs: cheaper barriers,
    // more rows per thread).
    if (const char* cap = std::getenv("RSATB_PERSIST_CTAS")) {
        const int64_t c = std::atoll(cap);
        if (c > 0 && c < grid) grid = c;
    }
    if (grid < 1) grid = 1;
    if (size_t(pa.n_steps + 1) * size_t(grid) * 2 * pa.base.W > part_capacity)
        return kPersistSkipped;  // the caller's slots were sized for fewer CTAs
    RSATB_CUDA_TRY(cudaMemsetAsync(pa.bar, 0, sizeof(unsigned), ctx->stream));
    void* args[] = {&pa};
    RSATB_CUDA_TRY(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel),
                                               dim3(unsigned(grid)), dim3(threads), args, 0,
                                               ctx->stream));
    const int64_t n = int64_t(pa.n_steps + 1) * 2 * pa.base.W;
    const int rgrid = int(std::min<int64_t>((n + 255) / 256, int64_t(ctx->sm_count) * 4));
    persistent_dots_kernel<<<rgrid, 256, 0, ctx->stream>>>(pa.n_steps + 1, int(grid),
                                                          pa.base.W, pa.part, dots);
    RSATB_LAUNCH_CHECK(ctx);
    ctx->launches += 1;  // the cooperative launch (the check above counted the reduction)
    return RSATB_SUCCESS;
}

}  // namespace

// The persistent recurrence when it applies: a plain (orthogonal) operator
// with scalar blocks and real values, at most kPersistMaxValues panel values,
// a device that supports cooperative launches and RSATB_NO_PERSIST unset.
// *done = false (and nothing launched) otherwise.
int run_persistent_recurrence(rsatb_context* ctx, const rsatb_bsr_matrix* H, int vdt, int W,
                              double center, double inv_hw, int doubled, const void* psi,
                              void* const buf[3], int n_steps, double* part, size_t part_capacity,
                              double* dots, unsigned* bar, unsigned* fault, bool* done) {
    *done = false;
    constexpr int64_t kPersistMaxValues = int64_t(1) << 22;
    if (std::getenv("RSATB_NO_PERSIST") || std::getenv("RSATB_STEP_KERNEL")) return RSATB_SUCCESS;
    if (H->block_size != 1 || dtype_is_complex(H->dtype) || n_steps < 1) return RSATB_SUCCESS;
    if (dtype_is_double(H->dtype) != dtype_is_double(vdt)) return RSATB_SUCCESS;
    if (int64_t(H->n_block_rows) * W > kPersistMaxValues) return RSATB_SUCCESS;
    int coop = 0;
    RSATB_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->device));
    if (!coop) return RSATB_SUCCESS;
    const bool cv = dtype_is_complex(vdt), dbl = dtype_is_double(vdt);
    const int V = (W % 4 == 0) ? 4 : 2;
    if (W % V) return RSATB_SUCCESS;
    PersistArgs pa{};
    pa.base.n_block_rows = H->n_block_rows;
    pa.base.row_ptr = H->row_ptr;
    pa.base.col_ind = H->col_ind;
    pa.base.vals = H->values;
    pa.base.block_size = 1;
    pa.base.W = W;
    pa.base.s_in = 1.0;
    pa.base.c = center;
    pa.base.s_out = inv_hw;
    pa.base.imag = (H->flags & RSATB_BSR_IMAGINARY_UNIT) ? 1 : 0;
    pa.base.dot_mode = doubled ? DOT_DOUBLING : DOT_PLAIN;
    pa.base.psi0 = psi;
    pa.base.fault = fault;
    pa.psi = psi;
    for (int i = 0; i < 3; ++i) pa.buf[i] = buf[i];
    pa.n_steps = n_steps;
    pa.part = part;
    pa.bar = bar;
    const int64_t rows = H->n_block_rows;
    int st;
    if (dbl) {
        if (cv) st = V == 4 ? launch_persistent<double, 4, true>(ctx, pa, rows, dots, part_capacity)
                            : launch_persistent<double, 2, true>(ctx, pa, rows, dots, part_capacity);
        else st = V == 4 ? launch_persistent<double, 4, false>(ctx, pa, rows, dots, part_capacity)
                         : launch_persistent<double, 2, false>(ctx, pa, rows, dots, part_capacity);
    } else {
        if (cv) st = V == 4 ? launch_persistent<float, 4, true>(ctx, pa, rows, dots, part_capacity)
                            : launch_persistent<float, 2, true>(ctx, pa, rows, dots, part_capacity);
        else st = V == 4 ? launch_persistent<float, 4, false>(ctx, pa, rows, dots, part_capacity)
                         : launch_persistent<float, 2, false>(ctx, pa, rows, dots, part_capacity);
    }
    if (st == kPersistSkipped) return RSATB_SUCCESS;
    RSATB_TRY(st);
    *done = true;
    return RSATB_SUCCESS;
}

}  // namespace rsatb_b200
