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
// On the device: S P and H x are the fused BSR step kernels, S P with its
// column dots <p|Sp> fused into the step; the update of X and R computes
// alpha per column and the new <r|r> in the same launch; every dot is FP64
// and deterministic (fixed-order partial sums per CTA, then the last CTA
// over CTAs).  An iteration is three launches and one 8 x R-byte copy of
// the residuals, which the host reads one iteration behind for the stopping
// test.  With the graph-local factor Z (ISQRTMPreconditioner, whose
// type is Symmetric) the CG runs on Z^H S Z Y = Z^H B and X = Z Y.
#include "cheb_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace rsatb_b200 {

int run_step(rsatb_context* ctx, const rsatb_bsr_matrix* A, int vdt, const StepArgs& a);
int run_coldot(rsatb_context* ctx, int vdt, int64_t n_rows, const StepArgs& a);

namespace {

constexpr int kDotThreads = 256;
constexpr int kMaxCols = 256;  // columns a dot CTA covers at once

bool aligned16s(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Column c of a dot in the layout of the fused step kernels' dots: W real
// values per row, so a complex column is the pair (re, im) at 2c and a real
// one the value at c (imaginary part 0).
template <bool CV>
__device__ __forceinline__ double2 col_value(const double* d, int c) {
    if constexpr (CV) return make_double2(d[2 * c], d[2 * c + 1]);
    return make_double2(d[c], 0.0);
}

// X_c += alpha_c P_c, R_c -= alpha_c AP_c with alpha_c = rr_c / pap_c (0 for
// a converged column, |rr_c| < tol2, or a broken-down one, |pap_c| < 1e-14
// |rr_c|), and rr_out_c = <R_c|R_c> of the updated R: thread (sub, column)
// of a CTA walks every (subs x gridDim.x)-th row, the CTA sums its rows in
// a fixed order, and the last CTA to finish (ticket counter) sums the CTA
// partials in a fixed order and resets the counter.  Deterministic.
template <typename T, bool CV>
__global__ void __launch_bounds__(kDotThreads)
cg_update_kernel(T* __restrict__ X, const T* __restrict__ P, T* __restrict__ R,
                 const T* __restrict__ AP, const double* __restrict__ rr,
                 const double* __restrict__ pap, double tol2, int64_t n_rows, int ncols,
                 double* __restrict__ part, double* __restrict__ rr_out,
                 unsigned* __restrict__ counter) {
    __shared__ double red[kDotThreads];
    __shared__ unsigned ticket;
    const int subs = kDotThreads / ncols;
    const int col = threadIdx.x % ncols, sub = threadIdx.x / ncols;
    double acc = 0.0;
    if (sub < subs) {
        const double2 r2 = col_value<CV>(rr, col), q2 = col_value<CV>(pap, col);
        const double nr = hypot(r2.x, r2.y), np = hypot(q2.x, q2.y);
        double ar = 0.0, ai = 0.0;
        if (!(nr < tol2 || np < 1e-14 * nr)) {
            const double d = q2.x * q2.x + q2.y * q2.y;
            ar = (r2.x * q2.x + r2.y * q2.y) / d;
            ai = (r2.y * q2.x - r2.x * q2.y) / d;
        }
#pragma unroll 4
        for (int64_t r = int64_t(blockIdx.x) * subs + sub; r < n_rows;
             r += int64_t(gridDim.x) * subs) {
            if constexpr (CV) {
                const int64_t e = r * ncols + col;
                const double pr = P[2 * e], pi = P[2 * e + 1];
                const double qr = AP[2 * e], qi = AP[2 * e + 1];
                X[2 * e] = T(double(X[2 * e]) + (ar * pr - ai * pi));
                X[2 * e + 1] = T(double(X[2 * e + 1]) + (ar * pi + ai * pr));
                const T nr_ = T(double(R[2 * e]) - (ar * qr - ai * qi));
                const T ni_ = T(double(R[2 * e + 1]) - (ar * qi + ai * qr));
                R[2 * e] = nr_;
                R[2 * e + 1] = ni_;
                acc += double(nr_) * double(nr_) + double(ni_) * double(ni_);
            } else {
                const int64_t e = r * ncols + col;
                X[e] = T(double(X[e]) + ar * double(P[e]));
                const T v = T(double(R[e]) - ar * double(AP[e]));
                R[e] = v;
                acc += double(v) * double(v);
            }
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < ncols) {
        double t = 0.0;
        for (int q = 0; q < subs; ++q) t += red[q * ncols + threadIdx.x];
        part[int64_t(blockIdx.x) * ncols + threadIdx.x] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) ticket = atomicAdd(counter, 1u);
    __syncthreads();
    if (ticket != gridDim.x - 1) return;
    __threadfence();
    // Eight independent partial sums per thread, so eight L2 loads are in
    // flight at once (a single chain costs one L2 round trip per CTA).
    double t8[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (sub < subs) {
        unsigned g = sub;
        for (; g + 7 * subs < gridDim.x; g += 8 * subs) {
#pragma unroll
            for (int u = 0; u < 8; ++u) t8[u] += __ldcg(part + int64_t(g + u * subs) * ncols + col);
        }
        for (; g < gridDim.x; g += subs) t8[0] += __ldcg(part + int64_t(g) * ncols + col);
    }
    red[threadIdx.x] = ((t8[0] + t8[1]) + (t8[2] + t8[3])) + ((t8[4] + t8[5]) + (t8[6] + t8[7]));
    __syncthreads();
    if (threadIdx.x < ncols) {
        double u = 0.0;
        for (int q = 0; q < subs; ++q) u += red[q * ncols + threadIdx.x];
        if constexpr (CV) {
            rr_out[2 * threadIdx.x] = u;
            rr_out[2 * threadIdx.x + 1] = 0.0;
        } else {
            rr_out[threadIdx.x] = u;
        }
    }
    if (threadIdx.x == 0) *counter = 0u;  // ready for the next launch
}

// beta_c = rr_new_c / rr_old_c (0 when rr_old_c vanishes); P_c = R_c + beta_c P_c.
template <typename T, bool CV>
__global__ void cg_direction_kernel(T* __restrict__ P, const T* __restrict__ R,
                                    const double* __restrict__ rr_old,
                                    const double* __restrict__ rr_new, int64_t n_elems,
                                    int ncols) {
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n_elems;
         e += int64_t(gridDim.x) * blockDim.x) {
        const int c = int(e % ncols);
        const double2 o = col_value<CV>(rr_old, c), n = col_value<CV>(rr_new, c);
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

// Y += c X with the complex coefficient c = (cr, ci) over n complex values
// (cv), or Y += Re(c) X over n real values (Chebyshev's CoeffCast for a real
// scalar type, rsatb/calc/cheby.hpp:113-121).
template <typename T>
__global__ void coeff_axpy_kernel(int64_t n, bool cv, double cr, double ci,
                                  const T* __restrict__ X, T* __restrict__ Y) {
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
         e += int64_t(gridDim.x) * blockDim.x) {
        if (cv) {
            const double xr = double(X[2 * e]), xi = double(X[2 * e + 1]);
            Y[2 * e] = T(double(Y[2 * e]) + cr * xr - ci * xi);
            Y[2 * e + 1] = T(double(Y[2 * e + 1]) + cr * xi + ci * xr);
        } else {
            Y[e] = T(double(Y[e]) + cr * double(X[e]));
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
    // Dots in the step kernels' layout (W doubles per dot; see col_value).
    double* part;     // CTA partials, sm_count x 8 x 2 x W
    double* d_rr;
    double* d_rr2;
    double* d_pap;
    double* d_dot;    // [dot_slots][W]
    unsigned* counter;
    unsigned* fault;
    int grid;  // CTAs of the update kernel
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

// out[0..W) = per-column <A|B> in the step kernels' layout.
int dots(const SolveCall& s, const SolveWork& w, const void* A, const void* B, double* out) {
    StepArgs a{};
    a.W = s.W;
    a.x = A;
    a.in = B;
    a.partials = w.part;
    a.dots_out = out;
    a.counter = w.counter;
    a.fault = w.fault;
    return run_coldot(s.ctx, s.vdt, s.n_rows, a);
}

int coeff_axpy(const SolveCall& s, double cr, double ci, const void* X, void* Y) {
    const bool cv = dtype_is_complex(s.vdt);
    const int64_t n = s.n_rows * s.W / (cv ? 2 : 1);
    if (dtype_is_double(s.vdt))
        coeff_axpy_kernel<double><<<elem_grid(s, n), 256, 0, s.ctx->stream>>>(
            n, cv, cr, ci, static_cast<const double*>(X), static_cast<double*>(Y));
    else
        coeff_axpy_kernel<float><<<elem_grid(s, n), 256, 0, s.ctx->stream>>>(
            n, cv, cr, ci, static_cast<const float*>(X), static_cast<float*>(Y));
    RSATB_LAUNCH_CHECK(s.ctx);
    return RSATB_SUCCESS;
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
int update_t(const SolveCall& s, const SolveWork& w, void* X, const double* rr, double tol2,
             double* rr_out) {
    cg_update_kernel<T, CV><<<w.grid, kDotThreads, 0, s.ctx->stream>>>(
        static_cast<T*>(X), static_cast<const T*>(w.P), static_cast<T*>(w.R),
        static_cast<const T*>(w.AP), rr, w.d_pap, tol2, s.n_rows, s.ncols, w.part, rr_out,
        w.counter);
    RSATB_LAUNCH_CHECK(s.ctx);
    return RSATB_SUCCESS;
}

template <typename T, bool CV>
int direction_t(const SolveCall& s, const SolveWork& w, const double* rr_old,
                const double* rr_new) {
    const int64_t n = s.n_rows * s.ncols;
    cg_direction_kernel<T, CV><<<elem_grid(s, n), 256, 0, s.ctx->stream>>>(
        static_cast<T*>(w.P), static_cast<const T*>(w.R), rr_old, rr_new, n, s.ncols);
    RSATB_LAUNCH_CHECK(s.ctx);
    return RSATB_SUCCESS;
}

int update(const SolveCall& s, const SolveWork& w, void* X, const double* rr, double tol2,
           double* rr_out) {
    const bool cv = dtype_is_complex(s.vdt);
    if (dtype_is_double(s.vdt))
        return cv ? update_t<double, true>(s, w, X, rr, tol2, rr_out)
                  : update_t<double, false>(s, w, X, rr, tol2, rr_out);
    return cv ? update_t<float, true>(s, w, X, rr, tol2, rr_out)
              : update_t<float, false>(s, w, X, rr, tol2, rr_out);
}

int direction(const SolveCall& s, const SolveWork& w, const double* o, const double* n) {
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
// (SymPrecondMat::mult_dense, rsatb/calc/preconditioner.hpp:249-262).  With
// dot_out, the last step also writes <in|out> per column there.
int apply_A(const SolveCall& s, const SolveWork& w, const rsatb_bsr_matrix* S,
            const rsatb_bsr_matrix* Z, const rsatb_bsr_matrix* ZH, const void* in, void* out,
            double* dot_out = nullptr) {
    StepArgs last = plain_args(s.W, nullptr, out);
    last.fault = w.fault;
    if (dot_out) {
        last.dot_mode = DOT_PLAIN;
        last.psi0 = in;
        last.partials = w.part;
        last.dots_out = dot_out;
        last.counter = w.counter;
    }
    if (!Z) {
        last.in = in;
        return run_step(s.ctx, S, s.vdt, last);
    }
    RSATB_TRY(run_step(s.ctx, Z, s.vdt, plain_args(s.W, in, w.u1)));
    RSATB_TRY(run_step(s.ctx, S, s.vdt, plain_args(s.W, w.u1, w.u2)));
    last.in = w.u2;
    return run_step(s.ctx, ZH, s.vdt, last);
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
    double* rr = w.d_rr;
    double* rr_new = w.d_rr2;
    RSATB_TRY(dots(s, w, w.R, w.R, rr));
    // The column residuals of iteration k are copied to pinned memory and
    // read after iteration k + 1 has been queued, so the device never waits
    // for the host's test.  A column whose residual is below tol is frozen
    // by the alpha kernel (alpha = 0: X and R unchanged), so once every
    // column has converged the extra queued iteration changes nothing and
    // the result equals a test after every iteration.
    const bool cv = dtype_is_complex(s.vdt);
    const int dw = cv ? 2 * s.ncols : s.ncols;  // doubles per dot
    void* pin = nullptr;
    RSATB_TRY(ctx_pinned(s.ctx, 2 * sizeof(double) * dw, &pin));
    double* hbuf[2] = {static_cast<double*>(pin), static_cast<double*>(pin) + dw};
    cudaEvent_t ev[2];
    RSATB_CUDA_TRY(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    const cudaError_t e_ev = cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    if (e_ev != cudaSuccess) cudaEventDestroy(ev[0]);
    RSATB_CUDA_TRY(e_ev);
    struct EvG {
        cudaEvent_t* e;
        ~EvG() {
            cudaEventDestroy(e[0]);
            cudaEventDestroy(e[1]);
        }
    } evg{ev};
    int it = 0;
    double max_err = 0.0;
    bool done = false;
    auto read = [&](int k) -> int {  // the test of iteration k (already queued)
        RSATB_CUDA_TRY(cudaEventSynchronize(ev[k & 1]));
        max_err = 0.0;
        const double* h = hbuf[k & 1];
        for (int c = 0; c < s.ncols; ++c)
            max_err = std::max(max_err, std::sqrt(cv ? std::hypot(h[2 * c], h[2 * c + 1])
                                                     : std::fabs(h[c])));
        it = k + 1;
        done = !(max_err >= tol);  // converged (or NaN: stop and report it)
        return RSATB_SUCCESS;
    };
    for (int k = 0; k < max_iter && !done; ++k) {
        RSATB_TRY(apply_A(s, w, S, Z, ZH, w.P, w.AP, w.d_pap));
        RSATB_TRY(update(s, w, X, rr, tol * tol, rr_new));
        RSATB_CUDA_TRY(cudaMemcpyAsync(hbuf[k & 1], rr_new, sizeof(double) * dw,
                                       cudaMemcpyDeviceToHost, s.ctx->stream));
        RSATB_CUDA_TRY(cudaEventRecord(ev[k & 1], s.ctx->stream));
        RSATB_TRY(direction(s, w, rr, rr_new));
        std::swap(rr, rr_new);
        if (k > 0) RSATB_TRY(read(k - 1));
        if (!done && k + 1 == max_iter) RSATB_TRY(read(k));
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
                int extra_panels, SolveCall* s, SolveWork* w, void** panels, int dot_slots = 1) {
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
                                                         int64_t(ctx->sm_count) * 2)));
    // CTA partials of the fused step kernels' dots (at most sm_count x 8
    // CTAs, two dots of W values) and of the update kernel (grid x R).
    const size_t part_b =
        (sizeof(double) * std::max(size_t(ctx->sm_count) * 8 * 2 * s->W,
                                   size_t(w->grid) * n_vectors) + 255) & ~size_t(255);
    const size_t col_b = ((sizeof(double) * s->W) + 255) & ~size_t(255);
    const int n_panels = 8 + extra_panels;
    void* base = nullptr;
    RSATB_TRY(ctx_scratch(ctx, n_panels * vb + part_b + (3 + dot_slots) * col_b, &base));
    RSATB_TRY(ctx_counters(ctx, 1, &w->counter));
    RSATB_TRY(ctx_fault_word(ctx, &w->fault));
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
    w->part = reinterpret_cast<double*>(q);
    q += part_b;
    w->d_rr = reinterpret_cast<double*>(q);
    w->d_rr2 = reinterpret_cast<double*>(q + col_b);
    w->d_pap = reinterpret_cast<double*>(q + 2 * col_b);
    w->d_dot = reinterpret_cast<double*>(q + 3 * col_b);
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

// Y = scale * S^-1 V X (NORMAL: V X is the CG's target and initial guess)
// or scale * V S^-1 X (adjoint: the solve from zero), Chebyshev::apply_dual
// for the Solve form (rsatb/calc/cheby.hpp:270-287).
int solve_form_apply_dual(rsatb_context* ctx, const rsatb_cheb_op* op,
                          const rsatb_bsr_matrix* V, const void* X, void* Y, int n_vectors,
                          int vdt, double scale, bool adjoint) {
    RSATB_TRY(check_solve_op(op, vdt));
    RSATB_TRY(check_bsr(V, "V"));
    if (V->n_block_rows != op->H->n_block_rows || V->block_size != op->H->block_size)
        return set_error(RSATB_INVALID_ARGUMENT, "V and H sizes differ");
    SolveCall s{};
    SolveWork w{};
    void* t[1] = {nullptr};
    RSATB_TRY(solve_setup(ctx, op->S, vdt, n_vectors, 1, &s, &w, t));
    int iters = 0;
    double resid = 0.0;
    if (!adjoint) {
        RSATB_TRY(run_step(ctx, V, vdt, plain_args(s.W, X, Y)));  // Y = V X
        RSATB_CUDA_TRY(cudaMemcpyAsync(t[0], Y, s.vbytes, cudaMemcpyDeviceToDevice, ctx->stream));
        RSATB_TRY(cg_solve(s, w, op->S, op->Z, op->ZH, t[0], Y, op_tol(op), op_iters(op), &iters,
                           &resid));
    } else {
        RSATB_CUDA_TRY(cudaMemsetAsync(t[0], 0, s.vbytes, ctx->stream));
        RSATB_TRY(cg_solve(s, w, op->S, op->Z, op->ZH, X, t[0], op_tol(op), op_iters(op), &iters,
                           &resid));
        RSATB_TRY(run_step(ctx, V, vdt, plain_args(s.W, t[0], Y)));  // Y = V S^-1 X
    }
    return axpby(s, 0.0, X, scale, Y);
}

// Y = sum_n c_n T_n(Op~) X with Op~ = (S^-1 H - c) / hw, one CG per
// application (Chebyshev::propagate, rsatb/calc/cheby.hpp:399-441): each
// solve starts from the contents of its output panel, which after the
// rotation holds T_{n-3} (the first two from zero).
int solve_form_propagate(rsatb_context* ctx, const rsatb_cheb_op* op, const void* X, void* Y,
                         int n_vectors, int vdt, const double* coeffs, int n_coeffs) {
    RSATB_TRY(check_solve_op(op, vdt));
    SolveCall s{};
    SolveWork w{};
    void* t[3] = {nullptr, nullptr, nullptr};
    RSATB_TRY(solve_setup(ctx, op->S, vdt, n_vectors, 3, &s, &w, t));
    RSATB_CUDA_TRY(cudaMemcpyAsync(t[0], X, s.vbytes, cudaMemcpyDeviceToDevice, ctx->stream));
    RSATB_CUDA_TRY(cudaMemsetAsync(t[1], 0, s.vbytes, ctx->stream));
    RSATB_CUDA_TRY(cudaMemsetAsync(t[2], 0, s.vbytes, ctx->stream));
    RSATB_CUDA_TRY(cudaMemsetAsync(Y, 0, s.vbytes, ctx->stream));
    RSATB_TRY(coeff_axpy(s, coeffs[0], coeffs[1], t[0], Y));
    if (n_coeffs == 1) return RSATB_SUCCESS;
    int iters = 0;
    double resid = 0.0;
    RSATB_TRY(apply_solve(s, w, op, t[0], t[1], &iters, &resid));
    RSATB_TRY(coeff_axpy(s, coeffs[2], coeffs[3], t[1], Y));
    for (int n = 2; n < n_coeffs; ++n) {
        RSATB_TRY(apply_solve(s, w, op, t[1], t[2], &iters, &resid));
        RSATB_TRY(axpby(s, -1.0, t[0], 2.0, t[2]));
        RSATB_TRY(coeff_axpy(s, coeffs[2 * n], coeffs[2 * n + 1], t[2], Y));
        void* old0 = t[0];
        t[0] = t[1];
        t[1] = t[2];
        t[2] = old0;
    }
    return RSATB_SUCCESS;
}

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
    // One dot slot per moment on the device, read back once at the end.
    RSATB_TRY(solve_setup(ctx, op->S, vdt, n_vectors, 3, &s, &w, t, n_moments));
    const int R = n_vectors;
    const size_t slot = ((sizeof(double) * s.W) + 255) & ~size_t(255);
    auto record = [&](int n, const void* a, const void* b) -> int {
        return dots(s, w, a, b,
                    reinterpret_cast<double*>(reinterpret_cast<char*>(w.d_dot) + n * slot));
    };
    auto finish = [&]() -> int {
        std::vector<double> h(slot / sizeof(double) * size_t(n_moments));
        RSATB_CUDA_TRY(cudaMemcpyAsync(h.data(), w.d_dot, slot * size_t(n_moments),
                                       cudaMemcpyDeviceToHost, ctx->stream));
        RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        const bool cv = dtype_is_complex(vdt);
        for (int n = 0; n < n_moments; ++n) {
            const double* d = h.data() + n * (slot / sizeof(double));
            double sr = 0.0, si = 0.0;
            for (int c = 0; c < R; ++c) {
                const double re = cv ? d[2 * c] : d[c], im = cv ? d[2 * c + 1] : 0.0;
                sr += re;
                si += im;
                if (col_mu_out) {
                    col_mu_out[2 * (size_t(n) * R + c)] = re;
                    col_mu_out[2 * (size_t(n) * R + c) + 1] = im;
                }
            }
            mu_out[2 * n] = sr / R;
            mu_out[2 * n + 1] = si / R;
        }
        return RSATB_SUCCESS;
    };
    // t0 = psi, t1 = t2 = 0 (the first solves start from zero).
    RSATB_CUDA_TRY(cudaMemcpyAsync(t[0], psi, s.vbytes, cudaMemcpyDeviceToDevice, ctx->stream));
    RSATB_CUDA_TRY(cudaMemsetAsync(t[1], 0, s.vbytes, ctx->stream));
    RSATB_CUDA_TRY(cudaMemsetAsync(t[2], 0, s.vbytes, ctx->stream));
    RSATB_TRY(record(0, psi, psi));
    if (n_moments == 1) return finish();
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
    return finish();
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
