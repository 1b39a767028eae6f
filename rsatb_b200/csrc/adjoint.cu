// Adjoint (vector-Jacobian product) of the KPM moment recurrence: the
// gradient of f = sum_n dmu_n mu_n, mu_n = (1/R) sum_s psi_s^T T_n(A) psi_s,
// A = (H - c) / hw, with respect to every stored block value of H.  There
// is no counterpart in the reference (RSATB has no differentiation code);
// the forward recurrence is rsatb/calc/cheby.hpp:479-514 (compute_moments).
//
// With t_n = T_n(A) psi (t_0 = psi, t_1 = A t_0, t_{n+1} = 2 A t_n - t_{n-1})
// the adjoint vectors follow the transposed recurrence
//     lambda_n = a_n psi + 2 A lambda_{n+1} - lambda_{n+2},   a_n = dmu_n / R,
// from lambda_N = lambda_{N+1} = 0 (A is symmetric), and
//     df/dA = lambda_1 t_0^T + 2 sum_{n=1}^{N-2} lambda_{n+1} t_n^T,
// so df/dH_ij = (df/dA)_ij / hw on the stored pattern: a sampled dense-dense
// product (SDDMM) of the lambda and t panels.
//
// Sandwich form, A = (Z^T H Z - c) / hw (real H symmetric): with
// G = df/dA = sum_n w_n lambda_{n+1} t_n^T as above,
//     df/dH = Z G Z^T / hw                     (SDDMM of Z lambda and Z t),
//     df/dZ = H Z (G + G^T) / hw               (SDDMMs of H Z lambda with t
//                                               and of H Z t with lambda),
// each on the stored pattern of its matrix; the four Z / H Z images of a
// segment's panels are formed by plain SpMMs before its SDDMMs.
//
// Memory: t_n is recomputed in segments of C moments from checkpoints
// (t_{kC}, t_{kC-1}) kept by the forward pass (C ~ sqrt(N)), so the
// backward pass holds O(sqrt(N)) panels, not N.  Each backward step is one
// fused step kernel (the a_n psi term rides in its epilogue); each segment
// ends with one SDDMM launch over the C moments of the segment.
#include "cheb_kernels.cuh"

#include <cmath>
#include <vector>

namespace rsatb_b200 {

int run_step(rsatb_context* ctx, const rsatb_bsr_matrix* A, int vdt, const StepArgs& a);
int run_coldot(rsatb_context* ctx, int vdt, int64_t n_rows, const StepArgs& a);

namespace {

// grad[k][r][c] += sum_{n in seg, n <= n_last} w_n sum_s L[n][i b + r][s] T[n][j b + c][s]
// for every stored block k = (i, j): one warp per (block, row r), lanes over
// the samples s, all b columns at once; w_n = (n == 0 ? 1 : 2) * scale.
template <typename VT, int B>
__global__ void __launch_bounds__(256) sddmm_kernel(int n_block_rows, const int32_t* row_ptr,
                                                    const int32_t* col_ind, int R, int n0,
                                                    int len, int n_last, double scale,
                                                    const VT* L, const VT* T, int64_t panel,
                                                    double* grad) {
    const int lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    const int64_t total_warps = int64_t(gridDim.x) * warps;
    const int64_t nnzb = row_ptr[n_block_rows];
    // work item: (k, r), k over stored blocks (row order), r < B
    for (int64_t w = int64_t(blockIdx.x) * warps + (threadIdx.x >> 5); w < nnzb * B;
         w += total_warps) {
        const int64_t k = w / B;
        const int r = int(w % B);
        // block row of k: binary search in row_ptr
        int lo = 0, hi = n_block_rows;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (row_ptr[mid] <= k) lo = mid;
            else hi = mid;
        }
        const int64_t i = lo;
        const int64_t j = col_ind[k];
        double acc[B];
#pragma unroll
        for (int c = 0; c < B; ++c) acc[c] = 0.0;
        for (int q = 0; q < len; ++q) {
            const int n = n0 + q;
            if (n > n_last) break;
            const double wn = (n == 0 ? 1.0 : 2.0);
            const VT* lrow = L + int64_t(q) * panel + (i * B + r) * R;
            const VT* tbase = T + int64_t(q) * panel + j * B * R;
            for (int s = lane; s < R; s += 32) {
                const double lv = wn * double(lrow[s]);
#pragma unroll
                for (int c = 0; c < B; ++c) acc[c] = fma(lv, double(tbase[c * R + s]), acc[c]);
            }
        }
#pragma unroll
        for (int c = 0; c < B; ++c) {
            double v = acc[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            acc[c] = v;
        }
        if (lane == 0) {
            double* g = grad + (k * B + r) * B;
#pragma unroll
            for (int c = 0; c < B; ++c) g[c] += scale * acc[c];
        }
    }
}

template <typename VT>
int launch_sddmm(rsatb_context* ctx, const rsatb_bsr_matrix* H, int R, int n0, int len,
                 int n_last, double scale, const VT* L, const VT* T, int64_t panel,
                 double* grad) {
    const int64_t items = H->nnz_blocks * H->block_size;
    int64_t grid = (items + 7) / 8;
    if (grid > int64_t(ctx->sm_count) * 16) grid = int64_t(ctx->sm_count) * 16;
    if (grid < 1) grid = 1;
#define RSATB_SDDMM(BV)                                                                    \
    sddmm_kernel<VT, BV><<<unsigned(grid), 256, 0, ctx->stream>>>(                         \
        H->n_block_rows, H->row_ptr, H->col_ind, R, n0, len, n_last, scale, L, T, panel, grad)
    switch (H->block_size) {
        case 1: RSATB_SDDMM(1); break;
        case 2: RSATB_SDDMM(2); break;
        case 3: RSATB_SDDMM(3); break;
        case 4: RSATB_SDDMM(4); break;
        case 5: RSATB_SDDMM(5); break;
        case 8: RSATB_SDDMM(8); break;
        default:
            return set_error(RSATB_NOT_SUPPORTED, "gradient for block size %d not built",
                             H->block_size);
    }
#undef RSATB_SDDMM
    RSATB_LAUNCH_CHECK(ctx);
    return RSATB_SUCCESS;
}

StepArgs zero_args(int W) {
    StepArgs a{};
    a.W = W;
    a.s_in = 1.0;
    a.s_out = 1.0;
    a.s2 = 1.0;
    a.dot_mode = DOT_NONE;
    return a;
}

template <typename VT>
int vjp_impl(rsatb_context* ctx, const rsatb_cheb_op* op, const VT* psi, int R, int vdt, int M,
             const double* dmu, int C, double* mu_out, double* grad, double* grad_z,
             rsatb_adjoint_stats* stats) {
    const rsatb_bsr_matrix* H = op->H;
    const bool sandwich = op->form == RSATB_FORM_SANDWICH;
    const int b = H->block_size;
    const int64_t N = int64_t(H->n_block_rows) * b;
    const int W = R;
    const int64_t panel = N * R;
    const size_t pbytes = size_t(panel) * sizeof(VT);
    cudaStream_t st = ctx->stream;
    if (C <= 0) C = int(std::ceil(std::sqrt(double(M))));
    if (C > M) C = M;
    const int n_seg = (M + C - 1) / C;

    // Everything lives in the context's grow-only scratch (no per-call
    // cudaMalloc / cudaFree): checkpoints, the two segment buffers, three
    // adjoint panels, a zero panel, three forward panels, dots, partials.
    const size_t pal = (pbytes + 255) & ~size_t(255);
    const size_t max_ctas = size_t(ctx->sm_count) * 8;
    const size_t dots_b = (size_t(M) * W * sizeof(double) + 255) & ~size_t(255);
    const size_t part_b = (max_ctas * 2 * W * sizeof(double) + 255) & ~size_t(255);
    // sandwich: two step intermediates and the Z t, Z lambda, H Z t, H Z
    // lambda images of a segment
    const size_t n_extra = sandwich ? 2 + 4 * size_t(C) : 0;
    const size_t n_pan = 2 * size_t(n_seg) + 2 * size_t(C) + 3 + 1 + 3 + n_extra;
    void* sp = nullptr;
    RSATB_TRY(ctx_scratch(ctx, n_pan * pal + dots_b + part_b, &sp));
    char* base = static_cast<char*>(sp);
    unsigned* counter = nullptr;
    RSATB_TRY(ctx_counters(ctx, 1, &counter));
    VT* ck = reinterpret_cast<VT*>(base);
    VT* tseg = reinterpret_cast<VT*>(base + 2 * size_t(n_seg) * pal);
    VT* lseg = reinterpret_cast<VT*>(base + (2 * size_t(n_seg) + C) * pal);
    VT* lam = reinterpret_cast<VT*>(base + (2 * size_t(n_seg) + 2 * C) * pal);
    VT* zero = reinterpret_cast<VT*>(base + (2 * size_t(n_seg) + 2 * C + 3) * pal);
    VT* f = reinterpret_cast<VT*>(base + (2 * size_t(n_seg) + 2 * C + 4) * pal);
    VT* su = sandwich ? reinterpret_cast<VT*>(base + (2 * size_t(n_seg) + 2 * C + 7) * pal)
                      : nullptr;
    VT* sw = sandwich ? su + pal / sizeof(VT) : nullptr;
    VT* zt = sandwich ? sw + pal / sizeof(VT) : nullptr;       // C panels each
    VT* zl = sandwich ? zt + size_t(C) * (pal / sizeof(VT)) : nullptr;
    VT* hzt = sandwich ? zl + size_t(C) * (pal / sizeof(VT)) : nullptr;
    VT* hzl = sandwich ? hzt + size_t(C) * (pal / sizeof(VT)) : nullptr;
    double* dots = reinterpret_cast<double*>(base + n_pan * pal);
    double* partials = reinterpret_cast<double*>(base + n_pan * pal + dots_b);
    RSATB_CUDA_TRY(cudaMemsetAsync(zero, 0, pbytes, st));
    RSATB_CUDA_TRY(cudaMemsetAsync(grad, 0, size_t(H->nnz_blocks) * b * b * sizeof(double), st));
    if (sandwich)
        RSATB_CUDA_TRY(cudaMemsetAsync(grad_z, 0,
                                       size_t(op->Z->nnz_blocks) * b * b * sizeof(double), st));

    const double inv_hw = 1.0 / op->half_width;
    auto step = [&](const VT* in, const VT* prev, VT* out, double s2, double g_p, const VT* q,
                    double g_q, double* dot_slot) -> int {
        StepArgs a = zero_args(W);
        a.in = in;
        a.x = in;
        a.p = prev;
        a.q = q;
        a.g_q = g_q;
        a.y = out;
        a.c = op->center;
        a.s_out = inv_hw;
        a.s2 = s2;
        a.g_p = g_p;
        if (dot_slot) {
            a.dot_mode = DOT_PLAIN;
            a.psi0 = psi;
            a.partials = partials;
            a.dots_out = dot_slot;
            a.counter = counter;
        }
        if (!sandwich) return run_step(ctx, H, vdt, a);
        StepArgs m = zero_args(W);  // su = Z in, sw = H su, then Z^T sw with the epilogue
        m.in = in;
        m.y = su;
        RSATB_TRY(run_step(ctx, op->Z, vdt, m));
        m.in = su;
        m.y = sw;
        RSATB_TRY(run_step(ctx, H, vdt, m));
        a.in = sw;
        return run_step(ctx, op->ZH, vdt, a);
    };
    auto mult = [&](const rsatb_bsr_matrix* A, const VT* in, VT* out) -> int {
        StepArgs m = zero_args(W);
        m.in = in;
        m.y = out;
        return run_step(ctx, A, vdt, m);
    };
    const size_t ps = pal / sizeof(VT);  // panel stride in elements
    auto ckpt = [&](int k, int which) { return ck + (2 * size_t(k) + which) * ps; };

    cudaEvent_t e0, e1, e2;
    RSATB_CUDA_TRY(cudaEventCreate(&e0));
    RSATB_CUDA_TRY(cudaEventCreate(&e1));
    RSATB_CUDA_TRY(cudaEventCreate(&e2));
    struct EvG {
        cudaEvent_t a, b, c;
        ~EvG() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
            cudaEventDestroy(c);
        }
    } evg{e0, e1, e2};
    RSATB_CUDA_TRY(cudaEventRecord(e0, st));

    // ---- forward: moments and checkpoints (t_{kC}, t_{kC-1})
    {
        StepArgs a = zero_args(W);
        a.x = psi;
        a.in = psi;
        a.partials = partials;
        a.dots_out = dots;
        a.counter = counter;
        RSATB_TRY(run_coldot(ctx, vdt, N, a));
    }
    const VT* tp = nullptr;  // t_{n-1}
    const VT* tc = psi;      // t_n
    int fs = 0;
    for (int n = 0; n < M; ++n) {
        if (n > 0) {
            VT* out = f + size_t(fs) * ps;
            fs = (fs + 1) % 3;
            if (n == 1) RSATB_TRY(step(tc, nullptr, out, 1.0, 0.0, nullptr, 0.0, dots + size_t(n) * W));
            else RSATB_TRY(step(tc, tp, out, 2.0, -1.0, nullptr, 0.0, dots + size_t(n) * W));
            tp = tc;
            tc = out;
        }
        if (n % C == 0) {
            const int k = n / C;
            RSATB_CUDA_TRY(cudaMemcpyAsync(ckpt(k, 0), tc, pbytes, cudaMemcpyDeviceToDevice, st));
            if (tp)
                RSATB_CUDA_TRY(cudaMemcpyAsync(ckpt(k, 1), tp, pbytes, cudaMemcpyDeviceToDevice, st));
        }
    }
    RSATB_CUDA_TRY(cudaEventRecord(e1, st));

    // ---- backward, segment by segment from the last
    const VT* l1 = zero;  // lambda_{n+1}
    const VT* l2 = zero;  // lambda_{n+2}
    int ls = 0;
    for (int k = n_seg - 1; k >= 0; --k) {
        const int nb0 = k * C;
        const int nb1 = std::min(M, nb0 + C);
        // recompute t_n, n in [nb0, nb1), into tseg
        RSATB_CUDA_TRY(cudaMemcpyAsync(tseg, ckpt(k, 0), pbytes, cudaMemcpyDeviceToDevice, st));
        for (int n = nb0 + 1; n < nb1; ++n) {
            VT* out = tseg + size_t(n - nb0) * ps;
            const VT* cur = tseg + size_t(n - 1 - nb0) * ps;
            if (n == 1) {
                RSATB_TRY(step(cur, nullptr, out, 1.0, 0.0, nullptr, 0.0, nullptr));
            } else {
                const VT* prv = (n - 2 >= nb0) ? tseg + size_t(n - 2 - nb0) * ps : ckpt(k, 1);
                RSATB_TRY(step(cur, prv, out, 2.0, -1.0, nullptr, 0.0, nullptr));
            }
        }
        for (int n = nb1 - 1; n >= nb0; --n) {
            // lambda_{n+1} pairs with t_n in the gradient
            RSATB_CUDA_TRY(cudaMemcpyAsync(lseg + size_t(n - nb0) * ps, l1, pbytes,
                                           cudaMemcpyDeviceToDevice, st));
            if (n >= 1) {
                VT* out = lam + size_t(ls) * ps;
                while (out == l1 || out == l2) {
                    ls = (ls + 1) % 3;
                    out = lam + size_t(ls) * ps;
                }
                ls = (ls + 1) % 3;
                RSATB_TRY(step(l1, l2, out, 2.0, -1.0, psi, dmu[n] / double(R), nullptr));
                l2 = l1;
                l1 = out;
            }
        }
        if (!sandwich) {
            RSATB_TRY(launch_sddmm<VT>(ctx, H, R, nb0, nb1 - nb0, M - 2, inv_hw, lseg, tseg,
                                       int64_t(ps), grad));
        } else {
            for (int q = 0; q < nb1 - nb0; ++q) {
                RSATB_TRY(mult(op->Z, tseg + size_t(q) * ps, zt + size_t(q) * ps));
                RSATB_TRY(mult(op->Z, lseg + size_t(q) * ps, zl + size_t(q) * ps));
                RSATB_TRY(mult(H, zt + size_t(q) * ps, hzt + size_t(q) * ps));
                RSATB_TRY(mult(H, zl + size_t(q) * ps, hzl + size_t(q) * ps));
            }
            RSATB_TRY(launch_sddmm<VT>(ctx, H, R, nb0, nb1 - nb0, M - 2, inv_hw, zl, zt,
                                       int64_t(ps), grad));
            RSATB_TRY(launch_sddmm<VT>(ctx, op->Z, R, nb0, nb1 - nb0, M - 2, inv_hw, hzl, tseg,
                                       int64_t(ps), grad_z));
            RSATB_TRY(launch_sddmm<VT>(ctx, op->Z, R, nb0, nb1 - nb0, M - 2, inv_hw, hzt, lseg,
                                       int64_t(ps), grad_z));
        }
    }
    RSATB_CUDA_TRY(cudaEventRecord(e2, st));

    std::vector<double> h(size_t(M) * W);
    RSATB_CUDA_TRY(cudaMemcpyAsync(h.data(), dots, h.size() * sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
    RSATB_CUDA_TRY(cudaStreamSynchronize(st));
    RSATB_TRY(ctx_check_fault(ctx));
    if (mu_out)
        for (int n = 0; n < M; ++n) {
            double s = 0.0;
            for (int q = 0; q < W; ++q) s += h[size_t(n) * W + q];
            mu_out[n] = s / double(R);
        }
    if (stats) {
        float a = 0.f, c = 0.f;
        cudaEventElapsedTime(&a, e0, e1);
        cudaEventElapsedTime(&c, e1, e2);
        stats->checkpoint_stride = C;
        stats->segments = n_seg;
        stats->forward_ms = a;
        stats->backward_ms = c;
        stats->panels_held = int(n_pan);
    }
    return RSATB_SUCCESS;
}

}  // namespace
}  // namespace rsatb_b200

using namespace rsatb_b200;

namespace {

int vjp_entry(rsatb_ctx_t ctx, const rsatb_cheb_op* op, const void* psi, int n_vectors,
              rsatb_dtype vec_dtype, int n_moments, const double* dmu, int checkpoint_stride,
              double* mu_out, double* grad_values, double* grad_z, rsatb_adjoint_stats* stats) {
    RSATB_TRY(check_ctx(ctx));
    if (!op || !psi || !dmu || !grad_values)
        return set_error(RSATB_INVALID_ARGUMENT, "null argument");
    RSATB_TRY(check_bsr(op->H, "H"));
    if (op->form == RSATB_FORM_SANDWICH) {
        RSATB_TRY(check_bsr(op->Z, "Z"));
        RSATB_TRY(check_bsr(op->ZH, "ZH"));
        if (!grad_z)
            return set_error(RSATB_INVALID_ARGUMENT, "the sandwich adjoint needs grad_z");
        if (op->Z->dtype != op->H->dtype || op->ZH->dtype != op->H->dtype ||
            op->Z->block_size != op->H->block_size ||
            op->Z->n_block_rows != op->H->n_block_rows || (op->Z->flags | op->ZH->flags))
            return set_error(RSATB_INVALID_ARGUMENT, "Z, Z^H and H differ in shape or type");
    }
    const rsatb_bsr_matrix* H = op->H;
    if (H->n_block_rows != H->n_block_cols)
        return set_error(RSATB_INVALID_ARGUMENT, "H must be square");
    if (dtype_is_complex(H->dtype) || dtype_is_complex(vec_dtype) ||
        (H->flags & RSATB_BSR_IMAGINARY_UNIT))
        return set_error(RSATB_NOT_SUPPORTED, "the adjoint takes a real H and real vectors");
    if (dtype_is_double(H->dtype) != dtype_is_double(vec_dtype))
        return set_error(RSATB_INVALID_ARGUMENT, "H and the vectors differ in precision");
    if (n_vectors <= 0 || n_vectors > 1536 || n_moments <= 0)
        return set_error(RSATB_INVALID_ARGUMENT, "bad n_vectors (%d) or n_moments (%d)", n_vectors,
                         n_moments);
    if (!(op->half_width > 0.0))
        return set_error(RSATB_INVALID_ARGUMENT, "half_width must be positive");
    if ((reinterpret_cast<uintptr_t>(psi) & 15u) != 0)
        return set_error(RSATB_INVALID_ARGUMENT, "psi must be 16-byte aligned");
    if (stats) *stats = rsatb_adjoint_stats{};
    if (dtype_is_double(vec_dtype))
        return vjp_impl<double>(ctx, op, static_cast<const double*>(psi), n_vectors,
                                int(vec_dtype), n_moments, dmu, checkpoint_stride, mu_out,
                                grad_values, grad_z, stats);
    return vjp_impl<float>(ctx, op, static_cast<const float*>(psi), n_vectors, int(vec_dtype),
                           n_moments, dmu, checkpoint_stride, mu_out, grad_values, grad_z,
                           stats);
}

}  // namespace

extern "C" int rsatb_kpm_moments_vjp(rsatb_ctx_t ctx, const rsatb_cheb_op* op, const void* psi,
                                     int n_vectors, rsatb_dtype vec_dtype, int n_moments,
                                     const double* dmu, int checkpoint_stride, double* mu_out,
                                     double* grad_values, rsatb_adjoint_stats* stats) {
    clear_error();
    if (ctx && op && op->form != RSATB_FORM_ORTHOGONAL)
        return set_error(RSATB_NOT_SUPPORTED,
                         "rsatb_kpm_moments_vjp runs the Orthogonal form; the sandwich form "
                         "is rsatb_kpm_moments_vjp_sandwich");
    return vjp_entry(ctx, op, psi, n_vectors, vec_dtype, n_moments, dmu, checkpoint_stride,
                     mu_out, grad_values, nullptr, stats);
}

extern "C" int rsatb_kpm_moments_vjp_sandwich(rsatb_ctx_t ctx, const rsatb_cheb_op* op,
                                              const void* psi, int n_vectors,
                                              rsatb_dtype vec_dtype, int n_moments,
                                              const double* dmu, int checkpoint_stride,
                                              double* mu_out, double* grad_h, double* grad_z,
                                              rsatb_adjoint_stats* stats) {
    clear_error();
    if (ctx && op && op->form != RSATB_FORM_SANDWICH)
        return set_error(RSATB_INVALID_ARGUMENT, "the operator is not in the sandwich form");
    return vjp_entry(ctx, op, psi, n_vectors, vec_dtype, n_moments, dmu, checkpoint_stride,
                     mu_out, grad_h, grad_z, stats);
}
