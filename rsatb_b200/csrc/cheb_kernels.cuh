// Fused BSR SpMM + Chebyshev step + FP64 column dots.
//
// One launch computes, for every row of the N x W output panel,
//
//     y = s2 * (((s_in * (A in)) - c * x) * s_out) + g_p * p [+ g_q * q]
//
// which covers BlockSpMat::mult_dense (s_in = alpha, no x, no p), the
// rescaled operator of Chebyshev::apply_form (rsatb/calc/cheby.hpp:555-591:
// y = A x; y -= c x; y *= 1/hw) and the recurrence t2 = 2 Op~ t1 - t0
// (rsatb/calc/dos.hpp:169-170), and accumulates in FP64 the per-column dots
// the KPM loop takes right after each step (dos.hpp:156-162):
//
//     DOT_DOUBLING   <y|x>, <y|y>      (the doubled recurrence)
//     DOT_PLAIN      <psi0|y>          (the plain recurrence)
//
// with <a|b> = sum_i conj(a_i) b_i per column.
//
// Layout: the panel is row-major with W real values per row (W = R for a
// real multivector, 2R for a complex one, (re, im) interleaved).  A thread
// owns V consecutive values of one block row; L = W / V threads share a
// block row and the CTA holds a whole number of such groups, so a
// grid-stride loop keeps each thread on the same columns and its dot partial sums stay in
// registers until one CTA-level reduction at the end.  The CTA partials go
// to global memory and the last CTA to finish sums them in CTA order, so the
// dots are deterministic for a given launch shape.
#pragma once

#include "common.cuh"

namespace rsatb_b200 {

enum DotMode { DOT_NONE = 0, DOT_DOUBLING = 1, DOT_PLAIN = 2 };

struct StepArgs {
    int64_t n_block_rows;
    const int32_t* row_ptr;
    const int32_t* col_ind;
    const void* vals;
    int block_size;    // runtime block size (generic kernel)
    int W;             // real values per row
    const void* in;    // SpMM operand
    const void* x;     // -c*x term and <y|x> partner (null: none)
    const void* p;     // recurrence predecessor (null: none)
    const void* psi0;  // DOT_PLAIN partner
    const void* q;     // optional extra term g_q * q (null: none)
    void* y;
    double s_in, c, s_out, s2, g_p, g_q;
    int imag;          // A = i * vals (real values, complex panel)
    int dot_mode;
    double* partials;  // [gridDim.x][ndots][W]
    double* dots_out;  // [ndots][W]
    unsigned* counter;
    unsigned* fault;   // set non-zero by a kernel whose bounded wait gave up (null: none)
    int wait_check;    // non-zero: the bulk-copy kernel only runs a wait that cannot
                       // complete (a 5 ms limit), to check the fault report
};

// Loads of V consecutive values.  CG = false: the read-only data path
// (__ldg), for data no thread of the launch writes; CG = true: L2-coherent
// loads (__ldcg), for data written earlier in the same launch.
template <typename T, bool CG>
__device__ __forceinline__ T ld_path(const T* p) {
    if constexpr (CG) return __ldcg(p);
    else return __ldg(p);
}

template <typename VT, int V, bool CG = false>
__device__ __forceinline__ void load_vals(const VT* __restrict__ p, VT (&o)[V]) {
    if constexpr (sizeof(VT) == 8 && V % 2 == 0) {
#pragma unroll
        for (int i = 0; i < V / 2; ++i) {
            const double2 t = ld_path<double2, CG>(reinterpret_cast<const double2*>(p) + i);
            o[2 * i] = t.x;
            o[2 * i + 1] = t.y;
        }
    } else if constexpr (sizeof(VT) == 4 && V % 4 == 0) {
#pragma unroll
        for (int i = 0; i < V / 4; ++i) {
            const float4 t = ld_path<float4, CG>(reinterpret_cast<const float4*>(p) + i);
            o[4 * i] = t.x;
            o[4 * i + 1] = t.y;
            o[4 * i + 2] = t.z;
            o[4 * i + 3] = t.w;
        }
    } else if constexpr (sizeof(VT) == 4 && V % 2 == 0) {
#pragma unroll
        for (int i = 0; i < V / 2; ++i) {
            const float2 t = ld_path<float2, CG>(reinterpret_cast<const float2*>(p) + i);
            o[2 * i] = t.x;
            o[2 * i + 1] = t.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < V; ++i) o[i] = ld_path<VT, CG>(p + i);
    }
}

template <typename VT, int V>
__device__ __forceinline__ void store_vals(VT* __restrict__ p, const VT (&o)[V]) {
    if constexpr (sizeof(VT) == 8 && V % 2 == 0) {
#pragma unroll
        for (int i = 0; i < V / 2; ++i)
            reinterpret_cast<double2*>(p)[i] = make_double2(o[2 * i], o[2 * i + 1]);
    } else if constexpr (sizeof(VT) == 4 && V % 4 == 0) {
#pragma unroll
        for (int i = 0; i < V / 4; ++i)
            reinterpret_cast<float4*>(p)[i] =
                make_float4(o[4 * i], o[4 * i + 1], o[4 * i + 2], o[4 * i + 3]);
    } else if constexpr (sizeof(VT) == 4 && V % 2 == 0) {
#pragma unroll
        for (int i = 0; i < V / 2; ++i)
            reinterpret_cast<float2*>(p)[i] = make_float2(o[2 * i], o[2 * i + 1]);
    } else {
#pragma unroll
        for (int i = 0; i < V; ++i) p[i] = o[i];
    }
}

// (d0, d1) += a * (b0, b1): one packed FP32 FMA (fma.rn.f32x2, sm_100),
// each lane an IEEE fused multiply-add, so the results equal two fmaf.
__device__ __forceinline__ void fma2(float& d0, float& d1, float a, float b0, float b1) {
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %2};\n\t"
        "mov.b64 rb, {%3, %4};\n\t"
        "mov.b64 rd, {%0, %1};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rd;\n\t"
        "mov.b64 {%0, %1}, rd;\n\t}"
        : "+f"(d0), "+f"(d1)
        : "f"(a), "f"(b0), "f"(b1));
}

// acc[v] += a * x[v] for v < V; FP32 with V even as packed pairs.
template <typename VT, int V>
__device__ __forceinline__ void fma_row(VT (&acc)[V], VT a, const VT (&x)[V]) {
    if constexpr (sizeof(VT) == 4 && V % 2 == 0) {
#pragma unroll
        for (int v = 0; v < V; v += 2) fma2(acc[v], acc[v + 1], a, x[v], x[v + 1]);
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = fma(a, x[v], acc[v]);
    }
}

// Epilogue for one output row: rescale, recurrence, store, dots.  CG: the
// x, p, q and psi0 panels are read through L2 (written earlier in the same
// launch).
template <typename VT, int V, bool CV, bool CG = false>
__device__ __forceinline__ void finish_row(const StepArgs& a, int64_t row, int g,
                                           const VT (&acc)[V], double (&d0)[V],
                                           double (&d1)[V]) {
    const int64_t off = row * a.W + int64_t(g) * V;
    double t[V];
#pragma unroll
    for (int v = 0; v < V; ++v) t[v] = double(acc[v]);
    if (CV && a.imag) {
        // (i * W) applied: (re, im) -> (-im, re)
#pragma unroll
        for (int v = 0; v < V; v += 2) {
            const double re = t[v];
            t[v] = -t[v + 1];
            t[v + 1] = re;
        }
    }
    VT xv[V];
    if (a.x) {
        load_vals<VT, V, CG>(static_cast<const VT*>(a.x) + off, xv);
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v) xv[v] = VT(0);
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
        double u = t[v] * a.s_in;
        if (a.x) u = fma(-a.c, double(xv[v]), u);
        t[v] = u * a.s_out;
    }
    if (a.p) {
        VT pv[V];
        load_vals<VT, V, CG>(static_cast<const VT*>(a.p) + off, pv);
#pragma unroll
        for (int v = 0; v < V; ++v) t[v] = fma(a.s2, t[v], a.g_p * double(pv[v]));
    } else if (a.s2 != 1.0) {
#pragma unroll
        for (int v = 0; v < V; ++v) t[v] *= a.s2;
    }
    if (a.q) {
        VT qv[V];
        load_vals<VT, V, CG>(static_cast<const VT*>(a.q) + off, qv);
#pragma unroll
        for (int v = 0; v < V; ++v) t[v] = fma(a.g_q, double(qv[v]), t[v]);
    }
    VT yv[V];
#pragma unroll
    for (int v = 0; v < V; ++v) yv[v] = VT(t[v]);
    store_vals<VT, V>(static_cast<VT*>(a.y) + off, yv);

    if (a.dot_mode == DOT_DOUBLING) {
        // <y|x> and <y|y>, from the stored (rounded) y.
        if constexpr (CV) {
#pragma unroll
            for (int v = 0; v < V; v += 2) {
                const double yr = double(yv[v]), yi = double(yv[v + 1]);
                const double xr = double(xv[v]), xi = double(xv[v + 1]);
                d0[v] += yr * xr + yi * xi;
                d0[v + 1] += yr * xi - yi * xr;
                d1[v] += yr * yr + yi * yi;
            }
        } else {
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const double yr = double(yv[v]);
                d0[v] += yr * double(xv[v]);
                d1[v] += yr * yr;
            }
        }
    } else if (a.dot_mode == DOT_PLAIN) {
        VT qv[V];
        load_vals<VT, V, CG>(static_cast<const VT*>(a.psi0) + off, qv);
        if constexpr (CV) {
#pragma unroll
            for (int v = 0; v < V; v += 2) {
                const double qr = double(qv[v]), qi = double(qv[v + 1]);
                const double yr = double(yv[v]), yi = double(yv[v + 1]);
                d0[v] += qr * yr + qi * yi;
                d0[v + 1] += qr * yi - qi * yr;
            }
        } else {
#pragma unroll
            for (int v = 0; v < V; ++v) d0[v] += double(qv[v]) * double(yv[v]);
        }
    }
}

// After every CTA wrote its partial dots: the last CTA to arrive (ticket
// counter) sums the gridDim.x partials of each of the O = ndots * W outputs
// and resets the counter for the next launch.  With fewer outputs than
// threads, T = blockDim / O threads share an output (CTAs b = part, part + T,
// ...) and their sums are combined in part order; otherwise each thread takes
// whole outputs with eight independent accumulators, so the L2 loads of one
// output are in flight together.  The order is fixed for a given grid:
// deterministic dots.  Needs blockDim.x <= 256.
// CTAs of at most 256 threads (comb below), which every step kernel uses.
__device__ __forceinline__ void finish_partials(const StepArgs& a, int ndots) {
    __threadfence();
    __syncthreads();
    __shared__ unsigned ticket;
    __shared__ double comb[256];
    if (threadIdx.x == 0) ticket = atomicAdd(a.counter, 1u);
    __syncthreads();
    if (ticket != gridDim.x - 1) return;
    __threadfence();
    const int O = ndots * a.W;
    const int nt = blockDim.x;
    const unsigned G = gridDim.x;
    const double* P = a.partials;
    if (O * 2 > nt) {
        for (int idx = threadIdx.x; idx < O; idx += nt) {
            double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0, s6 = 0, s7 = 0;
            unsigned b = 0;
            for (; b + 8 <= G; b += 8) {
                s0 += __ldcg(P + size_t(b) * O + idx);
                s1 += __ldcg(P + size_t(b + 1) * O + idx);
                s2 += __ldcg(P + size_t(b + 2) * O + idx);
                s3 += __ldcg(P + size_t(b + 3) * O + idx);
                s4 += __ldcg(P + size_t(b + 4) * O + idx);
                s5 += __ldcg(P + size_t(b + 5) * O + idx);
                s6 += __ldcg(P + size_t(b + 6) * O + idx);
                s7 += __ldcg(P + size_t(b + 7) * O + idx);
            }
            for (; b < G; ++b) s0 += __ldcg(P + size_t(b) * O + idx);
            a.dots_out[idx] = ((s0 + s1) + (s2 + s3)) + ((s4 + s5) + (s6 + s7));
        }
    } else {
        const int T = nt / O;
        const int o = threadIdx.x % O, part = threadIdx.x / O;
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        if (part < T) {
            unsigned b = part;
            for (; b + 3 * T < G; b += 4 * T) {
                s0 += __ldcg(P + size_t(b) * O + o);
                s1 += __ldcg(P + size_t(b + T) * O + o);
                s2 += __ldcg(P + size_t(b + 2 * T) * O + o);
                s3 += __ldcg(P + size_t(b + 3 * T) * O + o);
            }
            for (; b < G; b += T) s0 += __ldcg(P + size_t(b) * O + o);
        }
        comb[threadIdx.x] = (s0 + s1) + (s2 + s3);
        __syncthreads();
        if (threadIdx.x < O) {
            double t = 0.0;
            for (int q = 0; q < T; ++q) t += comb[q * O + threadIdx.x];
            a.dots_out[threadIdx.x] = t;
        }
    }
    if (threadIdx.x == 0) *a.counter = 0u;  // ready for the next launch
}

// CTA reduction of the per-thread dot partials, then the last-CTA
// reduction over CTAs.  Deterministic: fixed summation order throughout.
template <int V>
__device__ __forceinline__ void reduce_dots(const StepArgs& a, int L, const double (&d0)[V],
                                            const double (&d1)[V]) {
    extern __shared__ double red[];  // [ndots][blockDim.x][V]
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
        for (int t = g; t < nt; t += L) s += red[(d * nt + t) * V + v];
        mine[idx] = s;
    }
    finish_partials(a, ndots);
}

// Compile-time block size B.  MT: real component type of the matrix values;
// CM: complex matrix values; CV: complex panel.
template <typename VT, typename MT, int B, int V, bool CM, bool CV>
__global__ void __launch_bounds__(256) cheb_step_kernel(StepArgs a) {
    static_assert(!CM || CV, "a complex matrix needs a complex panel");
    static_assert(!CV || V % 2 == 0, "complex panels need (re, im) pairs per thread");
    const int L = a.W / V;
    const int g = threadIdx.x % L;
    const int64_t total = a.n_block_rows * L;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const MT* __restrict__ vals = static_cast<const MT*>(a.vals);
    const VT* __restrict__ in = static_cast<const VT*>(a.in);
    constexpr int BB = B * B * (CM ? 2 : 1);

    double d0[V], d1[V];
#pragma unroll
    for (int v = 0; v < V; ++v) d0[v] = d1[v] = 0.0;

    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += stride) {
        const int64_t i = t / L;
        VT acc[B][V];
#pragma unroll
        for (int r = 0; r < B; ++r)
#pragma unroll
            for (int v = 0; v < V; ++v) acc[r][v] = VT(0);
        const int k0 = __ldg(a.row_ptr + i), k1 = __ldg(a.row_ptr + i + 1);
        for (int k = k0; k < k1; ++k) {
            const int64_t j = __ldg(a.col_ind + k);
            // X_j: B rows x V values of this thread's columns.
            VT xb[B][V];
#pragma unroll
            for (int c = 0; c < B; ++c)
                load_vals<VT, V>(in + (j * B + c) * a.W + int64_t(g) * V, xb[c]);
            const MT* blk = vals + int64_t(k) * BB;
            constexpr int RW = B * (CM ? 2 : 1);  // values per block row
#pragma unroll
            for (int r = 0; r < B; ++r) {
                MT arow[RW];
                load_vals<MT, RW>(blk + r * RW, arow);
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
                        fma_row<VT, V>(acc[r], VT(arow[c]), xb[c]);
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < B; ++r)
            finish_row<VT, V, CV>(a, i * B + r, g, acc[r], d0, d1);
    }
    if (a.dot_mode != DOT_NONE) reduce_dots<V>(a, L, d0, d1);
}

// Runtime block size (b <= 16): the fallback for block sizes without a
// specialisation.  Same arithmetic, rows of the block handled one at a time.
template <typename VT, typename MT, int V, bool CM, bool CV>
__global__ void __launch_bounds__(256) cheb_step_kernel_any_b(StepArgs a) {
    const int L = a.W / V;
    const int g = threadIdx.x % L;
    const int B = a.block_size;
    const int64_t total = a.n_block_rows * L;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const MT* __restrict__ vals = static_cast<const MT*>(a.vals);
    const VT* __restrict__ in = static_cast<const VT*>(a.in);
    const int BB = B * B * (CM ? 2 : 1);

    double d0[V], d1[V];
#pragma unroll
    for (int v = 0; v < V; ++v) d0[v] = d1[v] = 0.0;

    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += stride) {
        const int64_t i = t / L;
        const int k0 = __ldg(a.row_ptr + i), k1 = __ldg(a.row_ptr + i + 1);
        for (int r = 0; r < B; ++r) {
            VT acc[V];
#pragma unroll
            for (int v = 0; v < V; ++v) acc[v] = VT(0);
            for (int k = k0; k < k1; ++k) {
                const int64_t j = __ldg(a.col_ind + k);
                const MT* blk = vals + int64_t(k) * BB;
                for (int c = 0; c < B; ++c) {
                    VT xv[V];
                    load_vals<VT, V>(in + (j * B + c) * a.W + int64_t(g) * V, xv);
                    if constexpr (CM) {
                        const VT ar = VT(__ldg(blk + 2 * (r * B + c)));
                        const VT ai = VT(__ldg(blk + 2 * (r * B + c) + 1));
#pragma unroll
                        for (int v = 0; v < V; v += 2) {
                            acc[v] = fma(ar, xv[v], acc[v]);
                            acc[v] = fma(-ai, xv[v + 1], acc[v]);
                            acc[v + 1] = fma(ar, xv[v + 1], acc[v + 1]);
                            acc[v + 1] = fma(ai, xv[v], acc[v + 1]);
                        }
                    } else {
                        const VT av = VT(__ldg(blk + r * B + c));
#pragma unroll
                        for (int v = 0; v < V; ++v) acc[v] = fma(av, xv[v], acc[v]);
                    }
                }
            }
            finish_row<VT, V, CV>(a, i * B + r, g, acc, d0, d1);
        }
    }
    if (a.dot_mode != DOT_NONE) reduce_dots<V>(a, L, d0, d1);
}

// Per-column <a|b> over n_rows rows (mu_0 = <psi|psi>), same reduction.
template <typename VT, int V, bool CV>
__global__ void __launch_bounds__(256) coldot_kernel(StepArgs a) {
    const int L = a.W / V;
    const int g = threadIdx.x % L;
    const int64_t total = a.n_block_rows * L;  // here: scalar rows
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    double d0[V], d1[V];
#pragma unroll
    for (int v = 0; v < V; ++v) d0[v] = d1[v] = 0.0;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += stride) {
        const int64_t row = t / L;
        const int64_t off = row * a.W + int64_t(g) * V;
        VT av[V], bv[V];
        load_vals<VT, V>(static_cast<const VT*>(a.x) + off, av);
        load_vals<VT, V>(static_cast<const VT*>(a.in) + off, bv);
        if constexpr (CV) {
#pragma unroll
            for (int v = 0; v < V; v += 2) {
                const double ar = double(av[v]), ai = double(av[v + 1]);
                const double br = double(bv[v]), bi = double(bv[v + 1]);
                d0[v] += ar * br + ai * bi;
                d0[v + 1] += ar * bi - ai * br;
            }
        } else {
#pragma unroll
            for (int v = 0; v < V; ++v) d0[v] += double(av[v]) * double(bv[v]);
        }
    }
    reduce_dots<V>(a, L, d0, d1);
}

// Launch entries for one fused step, defined per precision in
// cheb_step_f64.cu / cheb_step_f32.cu.
int launch_cheb_step_f64(rsatb_context* ctx, const rsatb_bsr_matrix* A, int vec_dtype,
                         StepArgs args);
int launch_cheb_step_f32(rsatb_context* ctx, const rsatb_bsr_matrix* A, int vec_dtype,
                         StepArgs args);
int launch_coldot_f64(rsatb_context* ctx, int vec_dtype, int64_t n_rows, StepArgs args);
int launch_coldot_f32(rsatb_context* ctx, int vec_dtype, int64_t n_rows, StepArgs args);

}  // namespace rsatb_b200
