// The Solve operator form, S^-1 H: one batched conjugate-gradient solve with
// the overlap S per operator application.
//
// rsatb::calc::LinearSolver::solve for a multivector (rsatb/calc/solver.hpp:
// 216-312): the columns are solved together, with per-column step lengths;
// a column whose residual is below tol freezes (alpha = 0), a breakdown
// |<p|Sp>| < 1e-14 |<r|r>| freezes it too, and the iteration stops when the
// largest column residual is below tol.  Chebyshev::apply_form's Solve
// branch (rsatb/calc/cheby.hpp:569-590): y = S^-1 (H x) with y's previous
// contents as the initial guess, then y = (y - center x) / half_width.  The
// KPM recurrence over this operator is the plain one (dos.hpp:172-187):
// S^-1 H is not Hermitian, so the doubling identity does not apply.
//
// On the device: S P and H x are the fused BSR step kernels with no
// epilogue; the per-column dots are FP64 and deterministic (fixed-order
// partial sums per CTA, then over CTAs); alpha and beta are formed on the
// device; the host reads the column residuals once per iteration for the
// stopping test.  With the graph-local factor Z (ISQRTMPreconditioner, whose
// type is Symmetric) the CG runs on Z^H S Z Y = Z^H B and X = Z Y.
#include "cheb_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace rsatb_b200 {

int run_step(rsatb_context* ctx, const rsatb_bsr_matrix* A, int vdt, const StepArgs& a);

namespace {

constexpr int kDotThreads = 256;
constexpr int kMaxCols = 256;  // columns a dot CTA covers at once

bool aligned16s(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// part[b][c] = sum over the rows CTA b takes of conj(A_rc) B_rc.
template <typename T, bool CV>
__global__ void __launch_bounds__(kDotThreads)
col_dot_partials(const T* __restrict__ A, const T* __restrict__ B, int64_t n_rows, int ncols,
                 double2* __restrict__ part) {
    __shared__ double2 red[kDotThreads];
    const int W = CV ? 2 * ncols : ncols;
    const int subs = kDotThreads / ncols;
    const int col = threadIdx.x % ncols, sub = threadIdx.x / ncols;
    double re = 0.0, im = 0.0;
    if (sub < subs) {
        for (int64_t r = int64_t(blockIdx.x) * subs + sub; r < n_rows;
             r += int64_t(gridDim.x) * subs) {
            if constexpr (CV) {
                const double ar = A[r * W + 2 * col], ai = A[r * W + 2 * col + 1];
                const double br = B[r * W + 2 * col], bi = B[r * W + 2 * col + 1];
                re += ar * br + ai * bi;
                im += ar * bi - ai * br;
            } else {
                re += double(A[r * W + col]) * double(B[r * W + col]);
            }
        }
    }
    red[threadIdx.x] = make_double2(re, im);
    __syncthreads();
    if (threadIdx.x < ncols) {
        double sr = 0.0, si = 0.0;
        for (int q = 0; q < subs; ++q) {
            sr += red[q * ncols + threadIdx.x].x;
            si += red[q * ncols + threadIdx.x].y;
        }
        part[int64_t(blockIdx.x) * ncols + threadIdx.x] = make_double2(sr, si);
    }
}

__global__ void col_dot_finish(const double2* __restrict__ part, int G, int ncols,
                               double2* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncols) return;
    double sr = 0.0, si = 0.0;
    for (int g = 0; g < G; ++g) {
        sr += part[int64_t(g) * ncols + c].x;
        si += part[int64_t(g) * ncols + c].y;
    }
    out[c] = make_double2(sr, si);
}

// alpha_c = rr_c / pap_c, or 0 for a converged or broken-down column.
__global__ void cg_alpha_kernel(const double2* __restrict__ rr, const double2* __restrict__ pap,
                                int ncols, double tol2, double2* __restrict__ alpha) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncols) return;
    const double nr = hypot(rr[c].x, rr[c].y), np = hypot(pap[c].x, pap[c].y);
    if (nr < tol2 || np < 1e-14 * nr) {
        alpha[c] = make_double2(0.0, 0.0);
        return;
    }
    const double d = pap[c].x * pap[c].x + pap[c].y * pap[c].y;
    alpha[c] = make_double2((rr[c].x * pap[c].x + rr[c].y * pap[c].y) / d,
                            (rr[c].y * pap[c].x - rr[c].x * pap[c].y) / d);
}

// X_c += alpha_c P_c, R_c -= alpha_c AP_c.  One thread per (row, column).
template <typename T, bool CV>
__global__ void cg_update_kernel(T* __restrict__ X, const T* __restrict__ P, T* __restrict__ R,
                                 const T* __restrict__ AP, const double2* __restrict__ alpha,
                                 int64_t n_elems, int ncols) {
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n_elems;
         e += int64_t(gridDim.x) * blockDim.x) {
        const double2 a = alpha[e % ncols];
        if constexpr (CV) {
            const double pr = P[2 * e], pi = P[2 * e + 1];
            const double qr = AP[2 * e], qi = AP[2 * e + 1];
            X[2 * e] = T(double(X[2 * e]) + (a.x * pr - a.y * pi));
            X[2 * e + 1] = T(double(X[2 * e + 1]) + (a.x * pi + a.y * pr));
            R[2 * e] = T(double(R[2 * e]) - (a.x * qr - a.y * qi));
            R[2 * e + 1] = T(double(R[2 * e + 1]) - (a.x * qi + a.y * qr));
        } else {
            X[e] = T(double(X[e]) + a.x * double(P[e]));
            R[e] = T(double(R[e]) - a.x * double(AP[e]));
        }
    }
}

// beta_c = rr_new_c / rr_old_c (0 when rr_old_c vanishes); P_c = R_c + beta_c P_c.
template <typename T, bool CV>
__global__ void cg_direction_kernel(T* __restrict__ P, const T* __restrict__ R,
                                    const double2* __restrict__ rr_old,
                                    const double2* __restrict__ rr_new, int64_t n_elems,
                                    int ncols) {
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n_elems;
         e += int64_t(gridDim.x) * blockDim.x) {
        const int c = int(e % ncols);
        const double2 o = rr_old[c], n = rr_new[c];
        double br = 0.0, bi = 0.0;
        if (hypot(o.x, o.y) >= 1e-300) {
            const double d = o.x * o.x + o.y * o.y;
            br = (n.x * o.x + n.y * o.y) / d;
            bi = (n.y * o.x - n.x * o.y) / d;
        }
        if constexpr (CV) {
            const double pr = P[2 * e], pi = P[2 * e + 1];
            P[2 * e] = T(double(R[2 * e]) + (br * pr - bi * pi));
            P[2 * e + 1] = T(double(R[2 * e + 1]) + (br * pi + bi * pr));
        } else {
            P[e] = T(double(R[e]) + br * double(P[e]));
        }
    }
}

// Y = a X + b Y over n real values.
template <typename T>
__global__ void panel_axpby_kernel(int64_t n, double a, const T* __restrict__ X, double b,
                                   T* __restrict__ Y) {
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
         e += int64_t(gridDim.x) * blockDim.x)
        Y[e] = T(a * double(X[e]) + b * double(Y[e]));
}

// Device buffers of one solve-form call, carved from the context scratch.
struct SolveWork {
    void* R;
    void* P;
    void* AP;
    void* tmp;
    void* u1;   // Z p (preconditioned operator)
    void* u2;   // S Z p
    void* Yp;   // solution of the preconditioned system
    void* Bp;   // its right-hand side Z^H b
    double2* part;
    double2* d_rr;
    double2* d_rr2;
    double2* d_pap;
    double2* d_alpha;
    double2* d_dot;
    int grid;  // dot CTAs
};

struct SolveCall {
    rsatb_context* ctx;
    int vdt;
    int64_t n_rows;
    int ncols;   // columns R
    int W;       // real values per row
    size_t vbytes;
};

unsigned elem_grid(const SolveCall& s, int64_t n) {
    return unsigned(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256,
                                                           int64_t(s.ctx->sm_count) * 8)));
}

template <typename T, bool CV>
int dots_t(const SolveCall& s, const SolveWork& w, const void* A, const void* B, double2* out) {
    col_dot_partials<T, CV><<<w.grid, kDotThreads, 0, s.ctx->stream>>>(
        static_cast<const T*>(A), static_cast<const T*>(B), s.n_rows, s.ncols, w.part);
    RSATB_LAUNCH_CHECK(s.ctx);
    col_dot_finish<<<(s.ncols + 127) / 128, 128, 0, s.ctx->stream>>>(w.part, w.grid, s.ncols, out);
    RSATB_LAUNCH_CHECK(s.ctx);
    return RSATB_SUCCESS;
}

int dots(const SolveCall& s, const SolveWork& w, const void* A, const void* B, double2* out) {
    const bool cv = dtype_is_complex(s.vdt);
    if (dtype_is_double(s.vdt))
        return cv ? dots_t<double, true>(s, w, A, B, out) : dots_t<double, false>(s, w, A, B, out);
    return cv ? dots_t<float, true>(s, w, A, B, out) : dots_t<float, false>(s, w, A, B, out);
}

int axpby(const SolveCall& s, double a, const void* X, double b, void* Y) {
    const int64_t n = s.n_rows * s.W;
    if (dtype_is_double(s.vdt))
        panel_axpby_kernel<double><<<elem_grid(s, n), 256, 0, s.ctx->stream>>>(
            n, a, static_cast<const double*>(X), b, static_cast<double*>(Y));
    else
        panel_axpby_kernel<float><<<elem_grid(s, n), 256, 0, s.ctx->stream>>>(
            n, a, static_cast<const float*>(X), b, static_cast<float*>(Y));
    RSATB_LAUNCH_CHECK(s.ctx);
    return RSATB_SUCCESS;
}

template <typename T, bool CV>
int update_t(const SolveCall& s, const SolveWork& w, void* X) {
    const int64_t n = s.n_rows * s.ncols;
    cg_update_kernel<T, CV><<<elem_grid(s, n), 256, 0, s.ctx->stream>>>(
        static_cast<T*>(X), static_cast<const T*>(w.P), static_cast<T*>(w.R),
        static_cast<const T*>(w.AP), w.d_alpha, n, s.ncols);
    RSATB_LAUNCH_CHECK(s.ctx);
    return RSATB_SUCCESS;
}

template <typename T, bool CV>
int direction_t(const SolveCall& s, const SolveWork& w, const double2* rr_old,
                const double2* rr_new) {
    const int64_t n = s.n_rows * s.ncols;
    cg_direction_kernel<T, CV><<<elem_grid(s, n), 256, 0, s.ctx->stream>>>(
        static_cast<T*>(w.P), static_cast<const T*>(w.R), rr_old, rr_new, n, s.ncols);
    RSATB_LAUNCH_CHECK(s.ctx);
    return RSATB_SUCCESS;
}

int update(const SolveCall& s, const SolveWork& w, void* X) {
    const bool cv = dtype_is_complex(s.vdt);
    if (dtype_is_double(s.vdt))
        return cv ? update_t<double, true>(s, w, X) : update_t<double, false>(s, w, X);
    return cv ? update_t<float, true>(s, w, X) : update_t<float, false>(s, w, X);
}

int direction(const SolveCall& s, const SolveWork& w, const double2* o, const double2* n) {
    const bool cv = dtype_is_complex(s.vdt);
    if (dtype_is_double(s.vdt))
        return cv ? direction_t<double, true>(s, w, o, n) : direction_t<double, false>(s, w, o, n);
    return cv ? direction_t<float, true>(s, w, o, n) : direction_t<float, false>(s, w, o, n);
}

StepArgs plain_args(int W, const void* in, void* y) {
    StepArgs a{};
    a.W = W;
    a.in = in;
    a.y = y;
    a.s_in = 1.0;
    a.c = 0.0;
    a.s_out = 1.0;
    a.s2 = 1.0;
    a.g_p = 0.0;
    a.dot_mode = DOT_NONE;
    return a;
}

// out = S in, or Z^H S Z in when a symmetric preconditioner Z is given
// (SymPrecondMat::mult_dense, rsatb/calc/preconditioner.hpp:249-262).
int apply_A(const SolveCall& s, const SolveWork& w, const rsatb_bsr_matrix* S,
            const rsatb_bsr_matrix* Z, const rsatb_bsr_matrix* ZH, const void* in, void* out) {
    if (!Z) return run_step(s.ctx, S, s.vdt, plain_args(s.W, in, out));
    RSATB_TRY(run_step(s.ctx, Z, s.vdt, plain_args(s.W, in, w.u1)));
    RSATB_TRY(run_step(s.ctx, S, s.vdt, plain_args(s.W, w.u1, w.u2)));
    return run_step(s.ctx, ZH, s.vdt, plain_args(s.W, w.u2, out));
}

// Batched CG for A X = B from X's contents (solver.hpp:216-312), A = S or
// Z^H S Z.
int cg_core(const SolveCall& s, const SolveWork& w, const rsatb_bsr_matrix* S,
            const rsatb_bsr_matrix* Z, const rsatb_bsr_matrix* ZH, const void* B, void* X,
            double tol, int max_iter, int* iters_out, double* resid_out) {
    // R = B - A X, P = R
    RSATB_TRY(apply_A(s, w, S, Z, ZH, X, w.AP));
    RSATB_CUDA_TRY(cudaMemcpyAsync(w.R, B, s.vbytes, cudaMemcpyDeviceToDevice, s.ctx->stream));
    RSATB_TRY(axpby(s, -1.0, w.AP, 1.0, w.R));
    RSATB_CUDA_TRY(cudaMemcpyAsync(w.P, w.R, s.vbytes, cudaMemcpyDeviceToDevice, s.ctx->stream));
    double2* rr = w.d_rr;
    double2* rr_new = w.d_rr2;
    RSATB_TRY(dots(s, w, w.R, w.R, rr));
    std::vector<double2> h(s.ncols);
    int it = 0;
    double max_err = 0.0;
    for (int k = 0; k < max_iter; ++k) {
        RSATB_TRY(apply_A(s, w, S, Z, ZH, w.P, w.AP));
        RSATB_TRY(dots(s, w, w.P, w.AP, w.d_pap));
        cg_alpha_kernel<<<(s.ncols + 127) / 128, 128, 0, s.ctx->stream>>>(rr, w.d_pap, s.ncols,
                                                                         tol * tol, w.d_alpha);
        RSATB_LAUNCH_CHECK(s.ctx);
        RSATB_TRY(update(s, w, X));
        RSATB_TRY(dots(s, w, w.R, w.R, rr_new));
        RSATB_CUDA_TRY(cudaMemcpyAsync(h.data(), rr_new, sizeof(double2) * s.ncols,
                                       cudaMemcpyDeviceToHost, s.ctx->stream));
        RSATB_CUDA_TRY(cudaStreamSynchronize(s.ctx->stream));
        max_err = 0.0;
        for (const double2& v : h) max_err = std::max(max_err, std::sqrt(std::hypot(v.x, v.y)));
        it = k + 1;
        if (!(max_err >= tol)) break;  // converged (or NaN: stop and report it)
        RSATB_TRY(direction(s, w, rr, rr_new));
        std::swap(rr, rr_new);
    }
    if (iters_out) *iters_out += it;
    if (resid_out) *resid_out = std::max(*resid_out, max_err);
    if (!std::isfinite(max_err))
        return set_error(RSATB_NUMERICAL_FAILURE, "cg: residual is not finite");
    return RSATB_SUCCESS;
}

// S X = B.  With Z: the explicitly symmetric-preconditioned system
// Z^H S Z Y = Z^H B from Y = 0, then X = Z Y (solver.hpp:329-338); X's
// contents are not used then.  Without: CG from X's contents.
int cg_solve(const SolveCall& s, const SolveWork& w, const rsatb_bsr_matrix* S,
             const rsatb_bsr_matrix* Z, const rsatb_bsr_matrix* ZH, const void* B, void* X,
             double tol, int max_iter, int* iters_out, double* resid_out) {
    if (!Z) return cg_core(s, w, S, nullptr, nullptr, B, X, tol, max_iter, iters_out, resid_out);
    RSATB_TRY(run_step(s.ctx, ZH, s.vdt, plain_args(s.W, B, w.Bp)));
    RSATB_CUDA_TRY(cudaMemsetAsync(w.Yp, 0, s.vbytes, s.ctx->stream));
    RSATB_TRY(cg_core(s, w, S, Z, ZH, w.Bp, w.Yp, tol, max_iter, iters_out, resid_out));
    return run_step(s.ctx, Z, s.vdt, plain_args(s.W, w.Yp, X));
}

int solve_setup(rsatb_context* ctx, const rsatb_bsr_matrix* S, int vdt, int n_vectors,
                int extra_panels, SolveCall* s, SolveWork* w, void** panels) {
    RSATB_TRY(check_bsr(S, "S"));
    if (S->n_block_rows != S->n_block_cols)
        return set_error(RSATB_INVALID_ARGUMENT, "S must be square");
    if (!dtype_valid(vdt)) return set_error(RSATB_INVALID_ARGUMENT, "bad multivector dtype %d", vdt);
    if (dtype_is_double(S->dtype) != dtype_is_double(vdt))
        return set_error(RSATB_INVALID_ARGUMENT, "S precision differs from the multivector's");
    if (dtype_is_complex(S->dtype) && !dtype_is_complex(vdt))
        return set_error(RSATB_INVALID_ARGUMENT, "S is complex but the multivector is real");
    if (n_vectors <= 0 || n_vectors > kMaxCols)
        return set_error(RSATB_NOT_SUPPORTED, "the CG takes 1 to %d columns (got %d)", kMaxCols,
                         n_vectors);
    s->ctx = ctx;
    s->vdt = vdt;
    s->n_rows = int64_t(S->n_block_rows) * S->block_size;
    s->ncols = n_vectors;
    s->W = n_vectors * (dtype_is_complex(vdt) ? 2 : 1);
    s->vbytes = size_t(s->n_rows) * s->W * dtype_real_size(vdt);
    const size_t vb = (s->vbytes + 255) & ~size_t(255);
    const int subs = kDotThreads / n_vectors;
    w->grid = int(std::max<int64_t>(1, std::min<int64_t>((s->n_rows + subs - 1) / subs,
                                                         int64_t(ctx->sm_count) * 4)));
    const size_t part_b = ((sizeof(double2) * size_t(w->grid) * n_vectors) + 255) & ~size_t(255);
    const size_t col_b = ((sizeof(double2) * n_vectors) + 255) & ~size_t(255);
    const int n_panels = 8 + extra_panels;
    void* base = nullptr;
    RSATB_TRY(ctx_scratch(ctx, n_panels * vb + part_b + 5 * col_b, &base));
    char* p = static_cast<char*>(base);
    w->R = p;
    w->P = p + vb;
    w->AP = p + 2 * vb;
    w->tmp = p + 3 * vb;
    w->u1 = p + 4 * vb;
    w->u2 = p + 5 * vb;
    w->Yp = p + 6 * vb;
    w->Bp = p + 7 * vb;
    for (int i = 0; i < extra_panels; ++i) panels[i] = p + (8 + i) * vb;
    char* q = p + n_panels * vb;
    w->part = reinterpret_cast<double2*>(q);
    q += part_b;
    w->d_rr = reinterpret_cast<double2*>(q);
    w->d_rr2 = reinterpret_cast<double2*>(q + col_b);
    w->d_pap = reinterpret_cast<double2*>(q + 2 * col_b);
    w->d_alpha = reinterpret_cast<double2*>(q + 3 * col_b);
    w->d_dot = reinterpret_cast<double2*>(q + 4 * col_b);
    return RSATB_SUCCESS;
}

int check_solve_op(const rsatb_cheb_op* op, int vdt) {
    RSATB_TRY(check_bsr(op->H, "H"));
    if (op->H->n_block_rows != op->H->n_block_cols)
        return set_error(RSATB_INVALID_ARGUMENT, "H must be square");
    if (!op->S) return set_error(RSATB_INVALID_ARGUMENT, "the Solve form needs S");
    RSATB_TRY(check_bsr(op->S, "S"));
    if (op->S->n_block_rows != op->H->n_block_rows || op->S->block_size != op->H->block_size)
        return set_error(RSATB_INVALID_ARGUMENT, "S and H shapes differ");
    if (dtype_is_double(op->H->dtype) != dtype_is_double(vdt) ||
        (dtype_is_complex(op->H->dtype) && !dtype_is_complex(vdt)))
        return set_error(RSATB_INVALID_ARGUMENT, "H and the multivector types do not match");
    if (!(op->half_width > 0.0) || !std::isfinite(op->center))
        return set_error(RSATB_INVALID_ARGUMENT, "spectral window needs half_width > 0");
    if ((op->Z == nullptr) != (op->ZH == nullptr))
        return set_error(RSATB_INVALID_ARGUMENT, "a preconditioned Solve form needs Z and ZH");
    if (op->Z) {
        RSATB_TRY(check_bsr(op->Z, "Z"));
        RSATB_TRY(check_bsr(op->ZH, "ZH"));
        if (op->Z->n_block_rows != op->H->n_block_rows || op->Z->block_size != op->H->block_size ||
            op->ZH->n_block_rows != op->H->n_block_rows || op->ZH->block_size != op->H->block_size ||
            dtype_is_double(op->Z->dtype) != dtype_is_double(vdt) ||
            dtype_is_double(op->ZH->dtype) != dtype_is_double(vdt))
            return set_error(RSATB_INVALID_ARGUMENT, "Z, ZH and H shapes or precisions differ");
    }
    if (op->cg_tol < 0.0 || op->cg_max_iter < 0)
        return set_error(RSATB_INVALID_ARGUMENT, "cg_tol and cg_max_iter must not be negative");
    return RSATB_SUCCESS;
}

double op_tol(const rsatb_cheb_op* op) { return op->cg_tol > 0.0 ? op->cg_tol : 1e-8; }
int op_iters(const rsatb_cheb_op* op) { return op->cg_max_iter > 0 ? op->cg_max_iter : 1000; }

// y = (S^-1 (H x) - center x) / half_width, with y's contents as the CG
// initial guess (cheby.hpp:576-589).
int apply_solve(const SolveCall& s, const SolveWork& w, const rsatb_cheb_op* op, const void* x,
                void* y, int* iters, double* resid) {
    RSATB_TRY(run_step(s.ctx, op->H, s.vdt, plain_args(s.W, x, w.tmp)));
    RSATB_TRY(cg_solve(s, w, op->S, op->Z, op->ZH, w.tmp, y, op_tol(op), op_iters(op), iters,
                       resid));
    return axpby(s, -op->center / op->half_width, x, 1.0 / op->half_width, y);
}

}  // namespace

// Entry points behind rsatb_cheb_apply_op and rsatb_kpm_dos_moments for
// the Solve form.
int solve_form_apply(rsatb_context* ctx, const rsatb_cheb_op* op, const void* X, void* Y,
                     int n_vectors, int vdt) {
    RSATB_TRY(check_solve_op(op, vdt));
    SolveCall s{};
    SolveWork w{};
    RSATB_TRY(solve_setup(ctx, op->S, vdt, n_vectors, 0, &s, &w, nullptr));
    int iters = 0;
    double resid = 0.0;
    return apply_solve(s, w, op, X, Y, &iters, &resid);
}

int solve_form_moments(rsatb_context* ctx, const rsatb_cheb_op* op, const void* psi,
                       int n_vectors, int vdt, int n_moments, double* mu_out,
                       double* col_mu_out) {
    RSATB_TRY(check_solve_op(op, vdt));
    SolveCall s{};
    SolveWork w{};
    void* t[3] = {nullptr, nullptr, nullptr};
    RSATB_TRY(solve_setup(ctx, op->S, vdt, n_vectors, 3, &s, &w, t));
    const int R = n_vectors;
    std::vector<double2> h(R);
    auto record = [&](int n, const void* a, const void* b) -> int {
        RSATB_TRY(dots(s, w, a, b, w.d_dot));
        RSATB_CUDA_TRY(cudaMemcpyAsync(h.data(), w.d_dot, sizeof(double2) * R,
                                       cudaMemcpyDeviceToHost, ctx->stream));
        RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        double sr = 0.0, si = 0.0;
        for (int c = 0; c < R; ++c) {
            sr += h[c].x;
            si += h[c].y;
            if (col_mu_out) {
                col_mu_out[2 * (size_t(n) * R + c)] = h[c].x;
                col_mu_out[2 * (size_t(n) * R + c) + 1] = h[c].y;
            }
        }
        mu_out[2 * n] = sr / R;
        mu_out[2 * n + 1] = si / R;
        return RSATB_SUCCESS;
    };
    // t0 = psi, t1 = t2 = 0 (the first solves start from zero).
    RSATB_CUDA_TRY(cudaMemcpyAsync(t[0], psi, s.vbytes, cudaMemcpyDeviceToDevice, ctx->stream));
    RSATB_CUDA_TRY(cudaMemsetAsync(t[1], 0, s.vbytes, ctx->stream));
    RSATB_CUDA_TRY(cudaMemsetAsync(t[2], 0, s.vbytes, ctx->stream));
    RSATB_TRY(record(0, psi, psi));
    if (n_moments == 1) return RSATB_SUCCESS;
    int iters = 0;
    double resid = 0.0;
    RSATB_TRY(apply_solve(s, w, op, t[0], t[1], &iters, &resid));
    RSATB_TRY(record(1, psi, t[1]));
    for (int n = 2; n < n_moments; ++n) {
        // t2 = 2 Op~ t1 - t0 (t2's contents, psi_{n-3}, start the solve),
        // then rotate (t0, t1, t2) <- (t1, t2, t0) as dos.hpp:182-185 swaps.
        RSATB_TRY(apply_solve(s, w, op, t[1], t[2], &iters, &resid));
        RSATB_TRY(axpby(s, -1.0, t[0], 2.0, t[2]));
        RSATB_TRY(record(n, psi, t[2]));
        void* old0 = t[0];
        t[0] = t[1];
        t[1] = t[2];
        t[2] = old0;
    }
    return RSATB_SUCCESS;
}

}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" int rsatb_cg_solve(rsatb_ctx_t ctx, rsatb_bsr_t S, rsatb_bsr_t Z, rsatb_bsr_t ZH,
                              const void* B, void* X, int n_vectors, rsatb_dtype vec_dtype,
                              double tol, int max_iter, int* iterations, double* max_residual) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!B || !X) return set_error(RSATB_INVALID_ARGUMENT, "null multivector");
    if (B == X) return set_error(RSATB_INVALID_ARGUMENT, "B and X must be distinct");
    if (!aligned16s(B) || !aligned16s(X))
        return set_error(RSATB_INVALID_ARGUMENT, "multivectors must be 16-byte aligned");
    if (!(tol > 0.0) || max_iter < 1)
        return set_error(RSATB_INVALID_ARGUMENT, "cg needs tol > 0 and max_iter >= 1");
    if ((Z == nullptr) != (ZH == nullptr))
        return set_error(RSATB_INVALID_ARGUMENT, "the preconditioner needs Z and ZH");
    SolveCall s{};
    SolveWork w{};
    RSATB_TRY(solve_setup(ctx, S, vec_dtype, n_vectors, 0, &s, &w, nullptr));
    if (Z) {
        RSATB_TRY(check_bsr(Z, "Z"));
        RSATB_TRY(check_bsr(ZH, "ZH"));
        if (Z->n_block_rows != S->n_block_rows || Z->block_size != S->block_size ||
            ZH->n_block_rows != S->n_block_rows || ZH->block_size != S->block_size ||
            Z->dtype != S->dtype || ZH->dtype != S->dtype)
            return set_error(RSATB_INVALID_ARGUMENT, "Z, ZH and S shapes or types differ");
    }
    int it = 0;
    double res = 0.0;
    RSATB_TRY(cg_solve(s, w, S, Z, ZH, B, X, tol, max_iter, &it, &res));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    RSATB_TRY(ctx_check_fault(ctx));
    if (iterations) *iterations = it;
    if (max_residual) *max_residual = res;
    return RSATB_SUCCESS;
}
