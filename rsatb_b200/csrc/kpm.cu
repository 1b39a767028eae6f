// Chebyshev operator application and the KPM moment recurrence
// (rsatb/calc/cheby.hpp apply_form, rsatb/calc/dos.hpp kpm_dos_moments),
// driven from the host, computed on the device.
#include "cheb_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <string>
#include <vector>

namespace rsatb_b200 {

int run_step(rsatb_context* ctx, const rsatb_bsr_matrix* A, int vdt, const StepArgs& a) {
    StepArgs b = a;
    if (!b.fault) RSATB_TRY(ctx_fault_word(ctx, &b.fault));
    return dtype_is_double(vdt) ? launch_cheb_step_f64(ctx, A, vdt, b)
                                : launch_cheb_step_f32(ctx, A, vdt, b);
}

int run_persistent_recurrence(rsatb_context* ctx, const rsatb_bsr_matrix* H, int vdt, int W,
                              double center, double inv_hw, int doubled, const void* psi,
                              void* const buf[3], int n_steps, double* part, size_t part_capacity,
                              double* dots, unsigned* bar, unsigned* fault, bool* done);

int solve_form_apply(rsatb_context* ctx, const rsatb_cheb_op* op, const void* X, void* Y,
                     int n_vectors, int vdt);
int solve_form_moments(rsatb_context* ctx, const rsatb_cheb_op* op, const void* psi,
                       int n_vectors, int vdt, int n_moments, double* mu_out,
                       double* col_mu_out);
int solve_form_apply_dual(rsatb_context* ctx, const rsatb_cheb_op* op,
                          const rsatb_bsr_matrix* V, const void* X, void* Y, int n_vectors,
                          int vdt, double scale, bool adjoint);
int solve_form_propagate(rsatb_context* ctx, const rsatb_cheb_op* op, const void* X, void* Y,
                         int n_vectors, int vdt, const double* coeffs, int n_coeffs);

int run_coldot(rsatb_context* ctx, int vdt, int64_t n_rows, const StepArgs& a) {
    return dtype_is_double(vdt) ? launch_coldot_f64(ctx, vdt, n_rows, a)
                                : launch_coldot_f32(ctx, vdt, n_rows, a);
}

namespace {

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

StepArgs blank_args(int W) {
    StepArgs a{};
    a.W = W;
    a.s_in = 1.0;
    a.c = 0.0;
    a.s_out = 1.0;
    a.s2 = 1.0;
    a.g_p = 0.0;
    a.dot_mode = DOT_NONE;
    return a;
}

struct OpShape {
    int64_t n_rows;  // scalar rows N
    bool sandwich;
};

int check_matrix_square(const rsatb_bsr_matrix* A, const char* name) {
    RSATB_TRY(check_bsr(A, name));
    if (A->n_block_rows != A->n_block_cols)
        return set_error(RSATB_INVALID_ARGUMENT, "%s must be square (%d x %d blocks)", name,
                         A->n_block_rows, A->n_block_cols);
    return RSATB_SUCCESS;
}

int check_vec_dtype(const rsatb_bsr_matrix* A, int vdt, const char* name) {
    if (!dtype_valid(vdt)) return set_error(RSATB_INVALID_ARGUMENT, "bad multivector dtype %d", vdt);
    if (dtype_is_double(A->dtype) != dtype_is_double(vdt))
        return set_error(RSATB_INVALID_ARGUMENT,
                         "%s precision (dtype %d) differs from the multivector's (dtype %d)", name,
                         A->dtype, vdt);
    if (dtype_is_complex(A->dtype) && !dtype_is_complex(vdt))
        return set_error(RSATB_INVALID_ARGUMENT, "%s is complex but the multivector is real", name);
    return RSATB_SUCCESS;
}

int check_op(const rsatb_cheb_op* op, int vdt, OpShape* shape) {
    if (!op) return set_error(RSATB_INVALID_ARGUMENT, "null operator");
    RSATB_TRY(check_matrix_square(op->H, "H"));
    RSATB_TRY(check_vec_dtype(op->H, vdt, "H"));
    if (!(op->half_width > 0.0) || !std::isfinite(op->half_width) || !std::isfinite(op->center))
        return set_error(RSATB_INVALID_ARGUMENT, "spectral window needs half_width > 0 (got %g)",
                         op->half_width);
    shape->n_rows = int64_t(op->H->n_block_rows) * op->H->block_size;
    if (op->form == RSATB_FORM_ORTHOGONAL) {
        shape->sandwich = false;
    } else if (op->form == RSATB_FORM_SANDWICH) {
        shape->sandwich = true;
        RSATB_TRY(check_matrix_square(op->Z, "Z"));
        RSATB_TRY(check_matrix_square(op->ZH, "ZH"));
        RSATB_TRY(check_vec_dtype(op->Z, vdt, "Z"));
        RSATB_TRY(check_vec_dtype(op->ZH, vdt, "ZH"));
        const int64_t nz = int64_t(op->Z->n_block_rows) * op->Z->block_size;
        const int64_t nzh = int64_t(op->ZH->n_block_rows) * op->ZH->block_size;
        if (nz != shape->n_rows || nzh != shape->n_rows)
            return set_error(RSATB_INVALID_ARGUMENT, "Z, Z^H and H sizes differ (%lld, %lld, %lld)",
                             (long long)nz, (long long)nzh, (long long)shape->n_rows);
    } else {
        return set_error(RSATB_NOT_SUPPORTED,
                         "operator form %d is not available on the device (the Solve form needs "
                         "a CG per matvec)", op->form);
    }
    return RSATB_SUCCESS;
}

int panel_width(int n_vectors, int vdt, int* W) {
    if (n_vectors <= 0) return set_error(RSATB_INVALID_ARGUMENT, "n_vectors must be positive");
    *W = n_vectors * (dtype_is_complex(vdt) ? 2 : 1);
    if (*W > 1536)
        return set_error(RSATB_NOT_SUPPORTED,
                         "%d vectors exceed the widest panel (1536 real values per row); split "
                         "the multivector", n_vectors);
    return RSATB_SUCCESS;
}

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

// y = ((Op) in - c x) * s_out * s2 + g_p * p with the dots of `dots`; `in`
// is the operand of the first factor (x itself for a plain application).
// u, w: sandwich intermediates.
int apply_fused(rsatb_context* ctx, const rsatb_cheb_op* op, const OpShape& sh, int vdt,
                int W, const void* in, const void* x, const void* p, void* y, void* u,
                void* w, double s_out, double s2, double g_p, int dot_mode, const void* psi0,
                double* partials, double* dots_out, unsigned* counter) {
    StepArgs last = blank_args(W);
    last.x = x;
    last.p = p;
    last.psi0 = psi0;
    last.y = y;
    last.c = op->center;
    last.s_out = s_out;
    last.s2 = s2;
    last.g_p = g_p;
    last.dot_mode = dot_mode;
    last.partials = partials;
    last.dots_out = dots_out;
    last.counter = counter;
    if (!sh.sandwich) {
        last.in = in;
        return run_step(ctx, op->H, vdt, last);
    }
    StepArgs a = blank_args(W);
    a.in = in;
    a.y = u;
    RSATB_TRY(run_step(ctx, op->Z, vdt, a));   // u = Z in
    a.in = u;
    a.y = w;
    RSATB_TRY(run_step(ctx, op->H, vdt, a));   // w = H u
    last.in = w;
    return run_step(ctx, op->ZH, vdt, last);   // y = Z^H w, fused epilogue
}


// Key of one recurrence launch sequence: every pointer and scalar its kernel
// arguments depend on.  A graph captured for a key replays only that key.
std::string recurrence_key(const rsatb_cheb_op* op, const void* psi, int n_vectors, int vdt,
                           int n_moments, int doubled, const void* scratch, const void* counter) {
    std::string k;
    auto put = [&](const void* p, size_t n) { k.append(static_cast<const char*>(p), n); };
    auto put_mat = [&](const rsatb_bsr_matrix* A) {
        put(&A, sizeof(A));
        if (!A) return;
        put(&A->values, sizeof(void*));
        put(&A->row_ptr, sizeof(void*));
        put(&A->col_ind, sizeof(void*));
        put(&A->nnz_blocks, sizeof(int64_t));
        put(&A->n_block_rows, sizeof(int));
        put(&A->block_size, sizeof(int));
        put(&A->dtype, sizeof(int));
        put(&A->flags, sizeof(unsigned));
    };
    put(&op->form, sizeof(int));
    put_mat(op->H);
    put_mat(op->form == RSATB_FORM_SANDWICH ? op->Z : nullptr);
    put_mat(op->form == RSATB_FORM_SANDWICH ? op->ZH : nullptr);
    put(&op->center, sizeof(double));
    put(&op->half_width, sizeof(double));
    put(&psi, sizeof(psi));
    put(&n_vectors, sizeof(int));
    put(&vdt, sizeof(int));
    put(&n_moments, sizeof(int));
    put(&doubled, sizeof(int));
    put(&scratch, sizeof(scratch));
    put(&counter, sizeof(counter));
    return k;
}

// Runs `issue` (the recurrence's launches) directly, or replays / captures
// it as a CUDA graph: a key seen on the previous call is captured once and
// then replayed while it stays the same, so a repeated call costs one graph
// launch instead of one host launch per step.  Graphs are off when the
// kernel choice is forced through the environment (its value is not part
// of the key) or RSATB_NO_GRAPH is set.  On the legacy default stream the
// graph runs on the context's own stream after the caller's queued work.
template <typename F>
int run_recurrence(rsatb_context* ctx, const rsatb_cheb_op* op, const void* psi, int n_vectors,
                   int vdt, int n_moments, int doubled, const void* scratch,
                   const void* counter, int n_steps, F&& issue) {
    const bool graph_ok = n_steps >= 8 && !std::getenv("RSATB_NO_GRAPH") &&
                          !std::getenv("RSATB_STEP_KERNEL") && !std::getenv("RSATB_STEP_V");
    if (!graph_ok) return issue();
    const std::string key =
        recurrence_key(op, psi, n_vectors, vdt, n_moments, doubled, scratch, counter);
    const bool replay = ctx->kpm_graph && ctx->kpm_graph_key == key;
    const bool capture = !replay && ctx->kpm_seen_key == key;
    if (!replay && !capture) {
        ctx->kpm_seen_key = key;
        return issue();
    }
    cudaStream_t run = ctx->stream ? ctx->stream : ctx->own_stream;
    if (run != ctx->stream) {
        cudaEvent_t e;
        RSATB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        const cudaError_t r1 = cudaEventRecord(e, ctx->stream);
        const cudaError_t r2 = cudaStreamWaitEvent(run, e, 0);
        cudaEventDestroy(e);
        RSATB_CUDA_TRY(r1);
        RSATB_CUDA_TRY(r2);
    }
    if (capture) {
        if (ctx->kpm_graph) {
            cudaGraphExecDestroy(ctx->kpm_graph);
            ctx->kpm_graph = nullptr;
            ctx->kpm_graph_key.clear();
        }
        cudaStream_t saved = ctx->stream;
        ctx->stream = run;
        const int64_t l0 = ctx->launches;
        RSATB_CUDA_TRY(cudaStreamBeginCapture(run, cudaStreamCaptureModeThreadLocal));
        const int st = issue();
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(run, &g);
        ctx->stream = saved;
        if (st != RSATB_SUCCESS) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (ec != cudaSuccess)
            return set_error(RSATB_CUDA_ERROR, "recurrence capture: %s", cudaGetErrorString(ec));
        const cudaError_t ei = cudaGraphInstantiate(&ctx->kpm_graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            ctx->kpm_graph = nullptr;
            return set_error(RSATB_CUDA_ERROR, "recurrence graph: %s", cudaGetErrorString(ei));
        }
        ctx->kpm_graph_key = key;
        ctx->kpm_graph_launches = ctx->launches - l0;
        ctx->launches = l0;
    }
    RSATB_CUDA_TRY(cudaGraphLaunch(ctx->kpm_graph, run));
    ctx->launches += ctx->kpm_graph_launches;
    if (run != ctx->stream) {
        // later work on the caller's stream sees the moments
        cudaEvent_t e;
        RSATB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        const cudaError_t r1 = cudaEventRecord(e, run);
        const cudaError_t r2 = cudaStreamWaitEvent(ctx->stream, e, 0);
        cudaEventDestroy(e);
        RSATB_CUDA_TRY(r1);
        RSATB_CUDA_TRY(r2);
    }
    return RSATB_SUCCESS;
}

// Y += c X over n complex (cv) or real values, c = (c_re, c_im); a real
// panel takes Re(c), as Chebyshev's CoeffCast does for a real scalar type
// (rsatb/calc/cheby.hpp:113-121).
template <typename T>
__global__ void axpy_coeff_kernel(int64_t n, bool cv, double c_re, double c_im, const T* X, T* Y) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    if (cv) {
        for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += stride) {
            const double xr = double(X[2 * i]), xi = double(X[2 * i + 1]);
            Y[2 * i] = T(double(Y[2 * i]) + c_re * xr - c_im * xi);
            Y[2 * i + 1] = T(double(Y[2 * i + 1]) + c_re * xi + c_im * xr);
        }
    } else {
        for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += stride)
            Y[i] = T(double(Y[i]) + c_re * double(X[i]));
    }
}

int axpy_coeff(rsatb_context* ctx, int vdt, int64_t n_values, double c_re, double c_im,
               const void* X, void* Y) {
    const bool cv = dtype_is_complex(vdt);
    const int64_t n = cv ? n_values / 2 : n_values;
    int64_t grid = (n + 255) / 256;
    if (grid > int64_t(ctx->sm_count) * 8) grid = int64_t(ctx->sm_count) * 8;
    if (grid < 1) grid = 1;
    if (dtype_is_double(vdt))
        axpy_coeff_kernel<double><<<unsigned(grid), 256, 0, ctx->stream>>>(
            n, cv, c_re, c_im, static_cast<const double*>(X), static_cast<double*>(Y));
    else
        axpy_coeff_kernel<float><<<unsigned(grid), 256, 0, ctx->stream>>>(
            n, cv, c_re, c_im, static_cast<const float*>(X), static_cast<float*>(Y));
    RSATB_LAUNCH_CHECK(ctx);
    return RSATB_SUCCESS;
}

}  // namespace
}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" {

int rsatb_bsr_mult_dense(rsatb_ctx_t ctx, rsatb_bsr_t A, const void* X, void* Y, int n_vectors,
                         rsatb_dtype vec_dtype, double alpha) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    RSATB_TRY(check_bsr(A, "A"));
    RSATB_TRY(check_vec_dtype(A, vec_dtype, "A"));
    int W = 0;
    RSATB_TRY(panel_width(n_vectors, vec_dtype, &W));
    if (!X || !Y) return set_error(RSATB_INVALID_ARGUMENT, "null multivector");
    if (!aligned16(X) || !aligned16(Y))
        return set_error(RSATB_INVALID_ARGUMENT, "multivectors must be 16-byte aligned");
    if (X == Y) return set_error(RSATB_INVALID_ARGUMENT, "mult_dense cannot run in place");
    StepArgs a = blank_args(W);
    a.in = X;
    a.y = Y;
    a.s_in = alpha;
    return run_step(ctx, A, vec_dtype, a);
}

int rsatb_cheb_apply_op(rsatb_ctx_t ctx, const rsatb_cheb_op* op, const void* X, void* Y,
                        int n_vectors, rsatb_dtype vec_dtype) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (op && op->form == RSATB_FORM_SOLVE) {
        if (!X || !Y) return set_error(RSATB_INVALID_ARGUMENT, "null multivector");
        if (!aligned16(X) || !aligned16(Y))
            return set_error(RSATB_INVALID_ARGUMENT, "multivectors must be 16-byte aligned");
        if (X == Y) return set_error(RSATB_INVALID_ARGUMENT, "apply_op cannot run in place");
        return solve_form_apply(ctx, op, X, Y, n_vectors, vec_dtype);
    }
    OpShape sh{};
    RSATB_TRY(check_op(op, vec_dtype, &sh));
    int W = 0;
    RSATB_TRY(panel_width(n_vectors, vec_dtype, &W));
    if (!X || !Y) return set_error(RSATB_INVALID_ARGUMENT, "null multivector");
    if (!aligned16(X) || !aligned16(Y))
        return set_error(RSATB_INVALID_ARGUMENT, "multivectors must be 16-byte aligned");
    if (X == Y) return set_error(RSATB_INVALID_ARGUMENT, "apply_op cannot run in place");
    const size_t vbytes = round256(size_t(sh.n_rows) * W * dtype_real_size(vec_dtype));
    void* u = nullptr;
    void* w = nullptr;
    if (sh.sandwich) {
        void* s = nullptr;
        RSATB_TRY(ctx_scratch(ctx, 2 * vbytes, &s));
        u = s;
        w = static_cast<char*>(s) + vbytes;
    }
    return apply_fused(ctx, op, sh, vec_dtype, W, X, X, nullptr, Y, u, w, 1.0 / op->half_width,
                       1.0, 0.0, DOT_NONE, nullptr, nullptr, nullptr, nullptr);
}

int rsatb_kpm_dos_moments(rsatb_ctx_t ctx, const rsatb_cheb_op* op, const void* psi,
                          int n_vectors, rsatb_dtype vec_dtype, int n_moments, int doubled,
                          double* mu_out, double* col_mu_out) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (op && op->form == RSATB_FORM_SOLVE) {
        if (n_moments <= 0) return set_error(RSATB_INVALID_ARGUMENT, "n_moments must be positive");
        if (!psi || !mu_out) return set_error(RSATB_INVALID_ARGUMENT, "null psi or mu_out");
        if (!aligned16(psi)) return set_error(RSATB_INVALID_ARGUMENT, "psi must be 16-byte aligned");
        if (doubled)
            return set_error(RSATB_INVALID_ARGUMENT,
                             "the Solve form S^-1 H is not Hermitian: use the plain recurrence "
                             "(doubled = 0)");
        RSATB_TRY(solve_form_moments(ctx, op, psi, n_vectors, vec_dtype, n_moments, mu_out,
                                     col_mu_out));
        RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        return ctx_check_fault(ctx);
    }
    OpShape sh{};
    RSATB_TRY(check_op(op, vec_dtype, &sh));
    int W = 0;
    RSATB_TRY(panel_width(n_vectors, vec_dtype, &W));
    if (n_moments <= 0) return set_error(RSATB_INVALID_ARGUMENT, "n_moments must be positive");
    if (!psi || !mu_out) return set_error(RSATB_INVALID_ARGUMENT, "null psi or mu_out");
    if (!aligned16(psi)) return set_error(RSATB_INVALID_ARGUMENT, "psi must be 16-byte aligned");
    const bool cv = dtype_is_complex(vec_dtype);
    const int R = n_vectors;

    // Number of operator applications.
    int n_steps = 0;
    if (n_moments > 1) {
        if (doubled) {
            n_steps = 1;
            for (int n = 1; 2 * n + 1 < n_moments; ++n) ++n_steps;
        } else {
            n_steps = n_moments - 1;
        }
    }
    const int ndots = doubled ? 2 : 1;

    // Scratch: three rotating panels, the sandwich pair, partial sums, dots.
    const size_t vbytes = round256(size_t(sh.n_rows) * W * dtype_real_size(vec_dtype));
    const size_t max_ctas = size_t(ctx->sm_count) * 8;
    const size_t part_bytes = round256(max_ctas * 2 * W * sizeof(double));
    const size_t dots_bytes = round256(size_t(n_steps + 1) * 2 * W * sizeof(double));
    const int n_panels = 3 + (sh.sandwich ? 2 : 0);
    // Per-step, per-CTA dot slots of the persistent recurrence (small
    // scalar-block operators; at most one CTA of 256 threads per 64 rows).
    const bool small_csr = !sh.sandwich && op->H->block_size == 1 && n_steps > 0 &&
                           int64_t(sh.n_rows) * W <= (int64_t(1) << 22);
    const size_t persist_grid =
        std::min<size_t>(size_t(ctx->sm_count) * 8, size_t(sh.n_rows) * W / 256 + 1);
    const size_t persist_elems = small_csr ? size_t(n_steps + 1) * persist_grid * 2 * W : 0;
    const size_t persist_bytes = round256(persist_elems * sizeof(double));
    const size_t total = n_panels * vbytes + part_bytes + dots_bytes + persist_bytes;
    void* s = nullptr;
    RSATB_TRY(ctx_scratch(ctx, total, &s));
    char* base = static_cast<char*>(s);
    void* buf[3] = {base, base + vbytes, base + 2 * vbytes};
    void* u = sh.sandwich ? base + 3 * vbytes : nullptr;
    void* w = sh.sandwich ? base + 4 * vbytes : nullptr;
    double* partials = reinterpret_cast<double*>(base + n_panels * vbytes);
    double* dots = reinterpret_cast<double*>(base + n_panels * vbytes + part_bytes);
    double* persist_part =
        reinterpret_cast<double*>(base + n_panels * vbytes + part_bytes + dots_bytes);
    unsigned* counter = nullptr;
    RSATB_TRY(ctx_counters(ctx, 2, &counter));
    unsigned* fault_word = nullptr;
    RSATB_TRY(ctx_fault_word(ctx, &fault_word));
    bool persistent = false;
    if (small_csr)
        RSATB_TRY(run_persistent_recurrence(ctx, op->H, vec_dtype, W, op->center,
                                            1.0 / op->half_width, doubled, psi, buf, n_steps,
                                            persist_part, persist_elems, dots, counter + 1,
                                            fault_word, &persistent));

    // The recurrence: mu_0 = <psi|psi> per column, then psi_1 = Op~ psi_0 and
    // psi_s = 2 Op~ psi_{s-1} - psi_{s-2}, each step with its fused dots.
    const double inv_hw = 1.0 / op->half_width;
    auto issue = [&]() -> int {
        {
            StepArgs a = blank_args(W);
            a.x = psi;
            a.in = psi;
            a.partials = partials;
            a.dots_out = dots;
            a.counter = counter;
            RSATB_TRY(run_coldot(ctx, vec_dtype, sh.n_rows, a));
        }
        const void* prev = nullptr;   // psi_{s-2}
        const void* cur = psi;        // psi_{s-1}
        int slot = 0;
        for (int sidx = 1; sidx <= n_steps; ++sidx) {
            void* out = buf[slot];
            slot = (slot + 1) % 3;
            double* dslot = dots + size_t(sidx) * 2 * W;
            RSATB_TRY(apply_fused(ctx, op, sh, vec_dtype, W, cur, cur, sidx == 1 ? nullptr : prev,
                                  out, u, w, inv_hw, sidx == 1 ? 1.0 : 2.0,
                                  sidx == 1 ? 0.0 : -1.0, doubled ? DOT_DOUBLING : DOT_PLAIN,
                                  psi, partials, dslot, counter));
            prev = cur;
            cur = out;
        }
        return RSATB_SUCCESS;
    };
    if (!persistent)
        RSATB_TRY(run_recurrence(ctx, op, psi, n_vectors, vec_dtype, n_moments, doubled, s,
                                 counter, n_steps, issue));

    std::vector<double> h(size_t(n_steps + 1) * 2 * W);
    RSATB_CUDA_TRY(cudaMemcpyAsync(h.data(), dots, sizeof(double) * h.size(),
                                   cudaMemcpyDeviceToHost, ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    RSATB_TRY(ctx_check_fault(ctx));

    using cd = std::complex<double>;
    // Per-column dot of slot s, dot d, column q.
    auto coldot = [&](int sidx, int d, int q) -> cd {
        const double* p = h.data() + size_t(sidx) * 2 * W + size_t(d) * W;
        return cv ? cd(p[2 * q], p[2 * q + 1]) : cd(p[q], 0.0);
    };
    // Per-column moments, then the column average in column order
    // (dos.hpp:134-138 averages the per-column dots the same way).
    std::vector<cd> colmu(size_t(n_moments) * R, cd(0.0, 0.0));
    for (int q = 0; q < R; ++q) {
        colmu[q] = coldot(0, 0, q);
        if (n_moments == 1) continue;
        if (doubled) {
            const cd mu0 = colmu[q];
            const cd mu1 = std::conj(coldot(1, 0, q));  // t0.dot(t1) = conj(<psi1|psi0>)
            colmu[size_t(1) * R + q] = mu1;
            for (int sidx = 1; sidx <= n_steps; ++sidx) {
                if (2 * sidx - 1 < n_moments && 2 * sidx - 1 > 1)
                    colmu[size_t(2 * sidx - 1) * R + q] = 2.0 * coldot(sidx, 0, q) - mu1;
                if (2 * sidx < n_moments)
                    colmu[size_t(2 * sidx) * R + q] = 2.0 * coldot(sidx, 1, q) - mu0;
            }
        } else {
            for (int sidx = 1; sidx <= n_steps; ++sidx)
                colmu[size_t(sidx) * R + q] = coldot(sidx, 0, q);
        }
    }
    for (int n = 0; n < n_moments; ++n) {
        cd sum(0.0, 0.0);
        if (doubled && n >= 1) {
            // mu_n = 2 * avg(d) - mu_{0 or 1}: average the dots first, as the
            // reference does, then apply the doubling formula.
            const int sidx = (n + 1) / 2;
            const bool odd = n % 2 == 1;
            cd dsum(0.0, 0.0);
            for (int q = 0; q < R; ++q) {
                if (n == 1) dsum += std::conj(coldot(1, 0, q));
                else dsum += coldot(sidx, odd ? 0 : 1, q);
            }
            const cd avg = dsum / double(R);
            if (n == 1) {
                sum = avg;
            } else {
                cd base(0.0, 0.0);
                for (int q = 0; q < R; ++q) base += odd ? std::conj(coldot(1, 0, q)) : coldot(0, 0, q);
                sum = 2.0 * avg - base / double(R);
            }
        } else {
            for (int q = 0; q < R; ++q) sum += colmu[size_t(n) * R + q];
            sum /= double(R);
        }
        mu_out[2 * n] = sum.real();
        mu_out[2 * n + 1] = sum.imag();
    }
    if (col_mu_out) {
        for (size_t i = 0; i < colmu.size(); ++i) {
            col_mu_out[2 * i] = colmu[i].real();
            col_mu_out[2 * i + 1] = colmu[i].imag();
        }
    }
    return RSATB_SUCCESS;
}

static int apply_dual_impl(rsatb_ctx_t ctx, const rsatb_cheb_op* op, rsatb_bsr_t V,
                           const void* X, void* Y, int n_vectors, rsatb_dtype vec_dtype,
                           double scale, bool adjoint) {
    RSATB_TRY(check_ctx(ctx));
    if (op && op->form == RSATB_FORM_SOLVE) {
        if (!X || !Y) return set_error(RSATB_INVALID_ARGUMENT, "null multivector");
        if (!aligned16(X) || !aligned16(Y))
            return set_error(RSATB_INVALID_ARGUMENT, "multivectors must be 16-byte aligned");
        if (X == Y) return set_error(RSATB_INVALID_ARGUMENT, "apply_dual cannot run in place");
        int W = 0;
        RSATB_TRY(panel_width(n_vectors, vec_dtype, &W));
        return solve_form_apply_dual(ctx, op, V, X, Y, n_vectors, vec_dtype, scale, adjoint);
    }
    OpShape sh{};
    RSATB_TRY(check_op(op, vec_dtype, &sh));
    RSATB_TRY(check_matrix_square(V, "V"));
    RSATB_TRY(check_vec_dtype(V, vec_dtype, "V"));
    if (int64_t(V->n_block_rows) * V->block_size != sh.n_rows)
        return set_error(RSATB_INVALID_ARGUMENT, "V and H sizes differ");
    int W = 0;
    RSATB_TRY(panel_width(n_vectors, vec_dtype, &W));
    if (!X || !Y) return set_error(RSATB_INVALID_ARGUMENT, "null multivector");
    if (!aligned16(X) || !aligned16(Y))
        return set_error(RSATB_INVALID_ARGUMENT, "multivectors must be 16-byte aligned");
    if (X == Y) return set_error(RSATB_INVALID_ARGUMENT, "apply_dual cannot run in place");
    StepArgs a = blank_args(W);
    if (!sh.sandwich) {
        a.in = X;
        a.y = Y;
        a.s_in = scale;
        return run_step(ctx, V, vec_dtype, a);
    }
    const size_t vbytes = round256(size_t(sh.n_rows) * W * dtype_real_size(vec_dtype));
    void* s = nullptr;
    RSATB_TRY(ctx_scratch(ctx, 2 * vbytes, &s));
    void* u = s;
    void* w = static_cast<char*>(s) + vbytes;
    a.in = X;
    a.y = u;
    RSATB_TRY(run_step(ctx, op->Z, vec_dtype, a));   // u = Z x
    a.in = u;
    a.y = w;
    RSATB_TRY(run_step(ctx, V, vec_dtype, a));       // w = V Z x
    a.in = w;
    a.y = Y;
    a.s_in = scale;
    return run_step(ctx, op->ZH, vec_dtype, a);      // y = scale Z^H V Z x
}

int rsatb_cheb_apply_dual(rsatb_ctx_t ctx, const rsatb_cheb_op* op, rsatb_bsr_t V,
                          const void* X, void* Y, int n_vectors, rsatb_dtype vec_dtype,
                          double scale) {
    clear_error();
    return apply_dual_impl(ctx, op, V, X, Y, n_vectors, vec_dtype, scale, false);
}

int rsatb_cheb_apply_dual_adjoint(rsatb_ctx_t ctx, const rsatb_cheb_op* op, rsatb_bsr_t V,
                                  const void* X, void* Y, int n_vectors, rsatb_dtype vec_dtype,
                                  double scale) {
    clear_error();
    return apply_dual_impl(ctx, op, V, X, Y, n_vectors, vec_dtype, scale, true);
}

int rsatb_cheb_propagate(rsatb_ctx_t ctx, const rsatb_cheb_op* op, const void* X, void* Y,
                         int n_vectors, rsatb_dtype vec_dtype, const double* coeffs,
                         int n_coeffs) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (op && op->form == RSATB_FORM_SOLVE) {
        if (n_coeffs < 0) return set_error(RSATB_INVALID_ARGUMENT, "n_coeffs < 0");
        if (n_coeffs == 0) return RSATB_SUCCESS;
        if (!X || !Y || !coeffs) return set_error(RSATB_INVALID_ARGUMENT, "null argument");
        if (!aligned16(X) || !aligned16(Y))
            return set_error(RSATB_INVALID_ARGUMENT, "multivectors must be 16-byte aligned");
        if (X == Y) return set_error(RSATB_INVALID_ARGUMENT, "propagate cannot run in place");
        int W = 0;
        RSATB_TRY(panel_width(n_vectors, vec_dtype, &W));
        return solve_form_propagate(ctx, op, X, Y, n_vectors, vec_dtype, coeffs, n_coeffs);
    }
    OpShape sh{};
    RSATB_TRY(check_op(op, vec_dtype, &sh));
    int W = 0;
    RSATB_TRY(panel_width(n_vectors, vec_dtype, &W));
    if (n_coeffs < 0) return set_error(RSATB_INVALID_ARGUMENT, "n_coeffs < 0");
    if (n_coeffs == 0) return RSATB_SUCCESS;  // Y unchanged, as the reference returns early
    if (!X || !Y || !coeffs) return set_error(RSATB_INVALID_ARGUMENT, "null argument");
    if (!aligned16(X) || !aligned16(Y))
        return set_error(RSATB_INVALID_ARGUMENT, "multivectors must be 16-byte aligned");
    if (X == Y) return set_error(RSATB_INVALID_ARGUMENT, "propagate cannot run in place");
    const int64_t n_values = sh.n_rows * W;
    const size_t vbytes = round256(size_t(n_values) * dtype_real_size(vec_dtype));
    const int n_panels = 3 + (sh.sandwich ? 2 : 0);
    void* s = nullptr;
    RSATB_TRY(ctx_scratch(ctx, n_panels * vbytes, &s));
    char* base = static_cast<char*>(s);
    void* buf[3] = {base, base + vbytes, base + 2 * vbytes};
    void* u = sh.sandwich ? base + 3 * vbytes : nullptr;
    void* w = sh.sandwich ? base + 4 * vbytes : nullptr;
    // Y = c_0 T_0 X = c_0 X (cheby.hpp:399-441): zero, then add.
    RSATB_CUDA_TRY(cudaMemsetAsync(Y, 0, size_t(n_values) * dtype_real_size(vec_dtype),
                                   ctx->stream));
    RSATB_TRY(axpy_coeff(ctx, vec_dtype, n_values, coeffs[0], coeffs[1], X, Y));
    const double inv_hw = 1.0 / op->half_width;
    const void* prev = nullptr;  // T_{n-2} X
    const void* cur = X;         // T_{n-1} X
    int slot = 0;
    for (int n = 1; n < n_coeffs; ++n) {
        void* out = buf[slot];
        slot = (slot + 1) % 3;
        // T_1 = Op~ X; T_n = 2 Op~ T_{n-1} - T_{n-2}
        RSATB_TRY(apply_fused(ctx, op, sh, vec_dtype, W, cur, cur, n == 1 ? nullptr : prev, out, u,
                              w, inv_hw, n == 1 ? 1.0 : 2.0, n == 1 ? 0.0 : -1.0, DOT_NONE,
                              nullptr, nullptr, nullptr, nullptr));
        RSATB_TRY(axpy_coeff(ctx, vec_dtype, n_values, coeffs[2 * n], coeffs[2 * n + 1], out, Y));
        prev = cur;
        cur = out;
    }
    return RSATB_SUCCESS;
}

}  // extern "C"
