// Extreme eigenvalues of the Chebyshev operator by Lanczos: the spectral
// window a Chebyshev<T> needs, which the reference takes from PRIMME
// (rsatb/setup/spectral_bounds.hpp:311-490, ExtremalEigenvalues with a
// residual tolerance of 1e-3 and the bounds_max_matvecs cap).
//
// The operator is applied unscaled (center 0, half width 1) through
// rsatb_cheb_apply_op, so every form is served: H, Z^H H Z, and S^-1 H with
// its CG, whose Lanczos basis is S-orthonormal (S^-1 H is self-adjoint in
// the S inner product: the generalised problem H x = lambda S x).  The
// basis is kept in FP64 (complex when the operator is), column-major with
// 16-byte aligned columns, and reorthogonalised twice per step against all
// earlier vectors (classical Gram-Schmidt, fixed-order FP64 dots: one CTA
// per basis vector).  The tridiagonal eigenproblem runs on the host by the
// implicit QL method with shifts (EISPACK's tql2: Bowdler, Martin, Reinsch
// and Wilkinson, Numer. Math. 11 (1968) 293-306), accumulating only the last
// row of the rotations: the Ritz values and the last components y_m of their
// vectors, whose |beta_m y_m| are the residual norms of the Ritz pairs.
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace rsatb_b200 {
namespace {

constexpr int kMaxKrylov = 400;   // basis vectors kept
constexpr int kDotThreads = 256;

// h[i] = sum_r conj(Q_i[r]) u[r] for i < k, as (re, im) pairs: CTA i sums
// column i in a fixed order (per-thread strided sums, then a shared tree).
template <bool CV>
__global__ void __launch_bounds__(kDotThreads)
basis_dots(const double* __restrict__ Q, int64_t ld, const double* __restrict__ u, int64_t n,
           double* __restrict__ h) {
    __shared__ double sr[kDotThreads], si[kDotThreads];
    const double* q = Q + int64_t(blockIdx.x) * ld;
    double re = 0.0, im = 0.0;
    for (int64_t r = threadIdx.x; r < n; r += kDotThreads) {
        if constexpr (CV) {
            const double qr = q[2 * r], qi = q[2 * r + 1];
            const double ur = u[2 * r], ui = u[2 * r + 1];
            re += qr * ur + qi * ui;
            im += qr * ui - qi * ur;
        } else {
            re += q[r] * u[r];
        }
    }
    sr[threadIdx.x] = re;
    si[threadIdx.x] = im;
    __syncthreads();
    for (int s = kDotThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sr[threadIdx.x] += sr[threadIdx.x + s];
            si[threadIdx.x] += si[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        h[2 * blockIdx.x] = sr[0];
        h[2 * blockIdx.x + 1] = si[0];
    }
}

// u[r] -= sum_{i < k} Q_i[r] h[i] (the sum in order of i).
template <bool CV>
__global__ void basis_subtract(const double* __restrict__ Q, int64_t ld, const double* __restrict__ h,
                               int k, int64_t n, double* __restrict__ u) {
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
         r += int64_t(gridDim.x) * blockDim.x) {
        if constexpr (CV) {
            double sr = 0.0, si = 0.0;
            for (int i = 0; i < k; ++i) {
                const double qr = Q[int64_t(i) * ld + 2 * r], qi = Q[int64_t(i) * ld + 2 * r + 1];
                sr += qr * h[2 * i] - qi * h[2 * i + 1];
                si += qr * h[2 * i + 1] + qi * h[2 * i];
            }
            u[2 * r] -= sr;
            u[2 * r + 1] -= si;
        } else {
            double s = 0.0;
            for (int i = 0; i < k; ++i) s += Q[int64_t(i) * ld + r] * h[2 * i];
            u[r] -= s;
        }
    }
}

// y = s x over m doubles.
__global__ void scale_copy(const double* __restrict__ x, double s, int64_t m, double* __restrict__ y) {
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < m;
         e += int64_t(gridDim.x) * blockDim.x)
        y[e] = s * x[e];
}

// FP64 <-> FP32 over m values (a panel of an FP32 operator).
__global__ void narrow_copy(const double* __restrict__ x, int64_t m, float* __restrict__ y) {
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < m;
         e += int64_t(gridDim.x) * blockDim.x)
        y[e] = float(x[e]);
}
__global__ void widen_copy(const float* __restrict__ x, int64_t m, double* __restrict__ y) {
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < m;
         e += int64_t(gridDim.x) * blockDim.x)
        y[e] = double(x[e]);
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

}  // namespace

// Eigenvalues (ascending) of the symmetric tridiagonal matrix with diagonal
// diag[0..m) and off-diagonal off[0..m-1), and the last component of each
// normalised eigenvector (the sign is arbitrary).  Implicit QL with shifts:
// for the leading unreduced block starting at l, the shift is the
// eigenvalue of its leading 2 x 2 block nearer d_l, and plane rotations
// chase the bulge from the bottom of the block up to l.
int tridiag_eigen(int m, const double* diag, const double* off, double* theta, double* last) {
    if (m <= 0) return RSATB_SUCCESS;
    std::vector<double> d(diag, diag + m), e(m, 0.0), z(m, 0.0);
    for (int i = 0; i + 1 < m; ++i) e[i] = off[i];  // e[i] couples i and i + 1
    z[m - 1] = 1.0;  // last row of the accumulated rotations
    const double eps = 2.220446049250313e-16;
    for (int l = 0; l < m; ++l) {
        for (int iter = 0;; ++iter) {
            int b = l;  // end of the unreduced block l..b
            while (b + 1 < m && std::fabs(e[b]) > eps * (std::fabs(d[b]) + std::fabs(d[b + 1]))) ++b;
            if (b == l) break;
            if (iter == 60)
                return set_error(RSATB_NUMERICAL_FAILURE,
                                 "tridiagonal QL did not converge at index %d", l);
            // Shift: eigenvalue of [[d_l, e_l], [e_l, d_l+1]] nearer d_l.
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[b] - d[l] + e[l] / (g + std::copysign(r, g));
            double s = 1.0, c = 1.0, p = 0.0;
            bool split = false;
            for (int i = b - 1; i >= l; --i) {
                const double f = s * e[i], h = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {  // the block splits here: restart on it
                    d[i + 1] -= p;
                    e[b] = 0.0;
                    split = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * h;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - h;
                const double zi = z[i], zi1 = z[i + 1];
                z[i + 1] = s * zi + c * zi1;
                z[i] = c * zi - s * zi1;
            }
            if (split) continue;
            d[l] -= p;
            e[l] = g;
            e[b] = 0.0;
        }
    }
    std::vector<int> order(m);
    for (int i = 0; i < m; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
    for (int i = 0; i < m; ++i) {
        theta[i] = d[order[i]];
        last[i] = z[order[i]];
    }
    return RSATB_SUCCESS;
}

}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" int rsatb_tridiag_eigen(int m, const double* diag, const double* off,
                                   double* eigenvalues, double* last_components) {
    clear_error();
    if (m < 0 || (m > 0 && (!diag || !eigenvalues || !last_components)) || (m > 1 && !off))
        return set_error(RSATB_INVALID_ARGUMENT, "bad tridiagonal arguments");
    return tridiag_eigen(m, diag, off, eigenvalues, last_components);
}

extern "C" int rsatb_lanczos_extremes(rsatb_ctx_t ctx, const rsatb_cheb_op* op,
                                      const rsatb_lanczos_options* options,
                                      rsatb_lanczos_result* result) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!op || !result) return set_error(RSATB_INVALID_ARGUMENT, "null operator or result");
    RSATB_TRY(check_bsr(op->H, "H"));
    if (op->H->n_block_rows != op->H->n_block_cols)
        return set_error(RSATB_INVALID_ARGUMENT, "H must be square");
    if (op->form == RSATB_FORM_SOLVE) RSATB_TRY(check_bsr(op->S, "S"));
    rsatb_lanczos_options o{};
    if (options) o = *options;
    const bool converge = o.tol > 0.0;
    const int max_mv = o.max_matvecs > 0 ? o.max_matvecs : 10000;
    const int steps = o.steps > 0 ? o.steps : 20;
    const int64_t n = int64_t(op->H->n_block_rows) * op->H->block_size;
    const bool cv = dtype_is_complex(op->H->dtype) || (op->H->flags & RSATB_BSR_IMAGINARY_UNIT);
    const bool f64 = dtype_is_double(op->H->dtype);
    const int vdt = f64 ? (cv ? RSATB_C128 : RSATB_F64) : (cv ? RSATB_C64 : RSATB_F32);
    const int wdt = cv ? RSATB_C128 : RSATB_F64;
    const bool solve = op->form == RSATB_FORM_SOLVE;
    int m = int(std::min<int64_t>(n, converge ? std::min(max_mv, kMaxKrylov) : steps));
    if (m < 1) m = 1;
    rsatb_cheb_op unit = *op;
    unit.center = 0.0;
    unit.half_width = 1.0;

    // Device buffers: Q (and S Q for the Solve form), m columns of ld
    // doubles; w (the matvec, FP64), t (S w), h (dots); an FP32 operator
    // also needs an FP32 input and output panel.
    const int64_t vals = cv ? 2 * n : n;         // doubles per vector
    const int64_t ld = (vals + 1) & ~int64_t(1);  // 16-byte aligned columns
    const size_t qbytes = sizeof(double) * size_t(ld) * size_t(m);
    DevBuf bq, bsq, bw, bt, bh, bx32, by32;
    RSATB_CUDA_TRY(cudaMalloc(&bq.p, qbytes));
    if (solve) RSATB_CUDA_TRY(cudaMalloc(&bsq.p, qbytes));
    RSATB_CUDA_TRY(cudaMalloc(&bw.p, sizeof(double) * size_t(ld)));
    RSATB_CUDA_TRY(cudaMalloc(&bt.p, sizeof(double) * size_t(ld)));
    RSATB_CUDA_TRY(cudaMalloc(&bh.p, sizeof(double) * 2 * size_t(m + 2)));
    if (!f64) {
        RSATB_CUDA_TRY(cudaMalloc(&bx32.p, sizeof(float) * size_t(ld)));
        RSATB_CUDA_TRY(cudaMalloc(&by32.p, sizeof(float) * size_t(ld)));
    }
    double* Q = static_cast<double*>(bq.p);
    double* SQ = solve ? static_cast<double*>(bsq.p) : Q;
    double* w = static_cast<double*>(bw.p);
    double* t = static_cast<double*>(bt.p);
    double* h = static_cast<double*>(bh.p);
    cudaStream_t st = ctx->stream;
    const unsigned eg = unsigned(std::min<int64_t>((vals + 255) / 256, int64_t(ctx->sm_count) * 8));

    auto dots = [&](const double* basis, int k, const double* u, double* out) -> int {
        if (cv) basis_dots<true><<<k, kDotThreads, 0, st>>>(basis, ld, u, n, out);
        else basis_dots<false><<<k, kDotThreads, 0, st>>>(basis, ld, u, n, out);
        RSATB_LAUNCH_CHECK(ctx);
        return RSATB_SUCCESS;
    };
    auto metric = [&](const double* x, double* out) -> int {  // out = S x (Solve form)
        if (f64) return rsatb_bsr_mult_dense(ctx, op->S, x, out, 1, rsatb_dtype(wdt), 1.0);
        narrow_copy<<<eg, 256, 0, st>>>(x, vals, static_cast<float*>(bx32.p));
        RSATB_LAUNCH_CHECK(ctx);
        RSATB_TRY(rsatb_bsr_mult_dense(ctx, op->S, bx32.p, by32.p, 1, rsatb_dtype(vdt), 1.0));
        widen_copy<<<eg, 256, 0, st>>>(static_cast<const float*>(by32.p), vals, out);
        RSATB_LAUNCH_CHECK(ctx);
        return RSATB_SUCCESS;
    };
    // s-norm squared of x: <x, S x> (or <x, x>), left in h[2 * slot].
    auto snorm2 = [&](const double* x, int slot) -> int {
        if (solve) {
            RSATB_TRY(metric(x, t));
            return dots(t, 1, x, h + 2 * slot);
        }
        return dots(x, 1, x, h + 2 * slot);
    };
    auto read = [&](int count, double* host) -> int {
        RSATB_CUDA_TRY(cudaMemcpyAsync(host, h, sizeof(double) * 2 * count, cudaMemcpyDeviceToHost, st));
        RSATB_CUDA_TRY(cudaStreamSynchronize(st));
        return RSATB_SUCCESS;
    };

    // Start vector: the seeded sample of rsatb_set_random (random phases,
    // or signs for a real operator), normalised in the S inner product.
    std::vector<int64_t> ids(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) ids[size_t(i)] = i;
    RSATB_TRY(rsatb_set_random(ctx, o.seed ? o.seed : 2, cv ? RSATB_RANDOM_PHASE : RSATB_RANDOM_RADEMACHER,
                               1, ids.data(), int(n), 1, n, 1, 0, rsatb_dtype(wdt), Q));
    RSATB_TRY(snorm2(Q, 0));
    double hv[4];
    RSATB_TRY(read(1, hv));
    if (!(hv[0] > 0.0) || !std::isfinite(hv[0]))
        return set_error(RSATB_NUMERICAL_FAILURE, "lanczos: the start vector has no S-norm");
    scale_copy<<<eg, 256, 0, st>>>(Q, 1.0 / std::sqrt(hv[0]), vals, Q);
    RSATB_LAUNCH_CHECK(ctx);

    std::vector<double> alpha(m, 0.0), beta(m, 0.0), th(m), yl(m);
    bool converged = !converge;
    int used = m;
    for (int j = 0; j < m; ++j) {
        double* qj = Q + int64_t(j) * ld;
        double* sqj = SQ + int64_t(j) * ld;
        if (solve) RSATB_TRY(metric(qj, sqj));
        // w = Op q (the Solve form's CG starts from w = 0)
        if (f64) {
            RSATB_CUDA_TRY(cudaMemsetAsync(w, 0, sizeof(double) * size_t(vals), st));
            RSATB_TRY(rsatb_cheb_apply_op(ctx, &unit, qj, w, 1, rsatb_dtype(vdt)));
        } else {
            narrow_copy<<<eg, 256, 0, st>>>(qj, vals, static_cast<float*>(bx32.p));
            RSATB_LAUNCH_CHECK(ctx);
            RSATB_CUDA_TRY(cudaMemsetAsync(by32.p, 0, sizeof(float) * size_t(vals), st));
            RSATB_TRY(rsatb_cheb_apply_op(ctx, &unit, bx32.p, by32.p, 1, rsatb_dtype(vdt)));
            widen_copy<<<eg, 256, 0, st>>>(static_cast<const float*>(by32.p), vals, w);
            RSATB_LAUNCH_CHECK(ctx);
        }
        // alpha_j = Re <S q_j, w>, kept at h[2 (m + 1)]
        RSATB_TRY(dots(sqj, 1, w, h + 2 * (m + 1)));
        for (int pass = 0; pass < 2; ++pass) {  // full reorthogonalisation
            RSATB_TRY(dots(SQ, j + 1, w, h));
            if (cv) basis_subtract<true><<<eg, 256, 0, st>>>(Q, ld, h, j + 1, n, w);
            else basis_subtract<false><<<eg, 256, 0, st>>>(Q, ld, h, j + 1, n, w);
            RSATB_LAUNCH_CHECK(ctx);
        }
        RSATB_TRY(snorm2(w, 0));
        RSATB_CUDA_TRY(cudaMemcpyAsync(hv + 2, h + 2 * (m + 1), sizeof(double) * 2,
                                       cudaMemcpyDeviceToHost, st));
        RSATB_TRY(read(1, hv));
        const double a = hv[2];
        const double b = std::sqrt(std::max(hv[0], 0.0));
        if (!std::isfinite(a) || !std::isfinite(b))
            return set_error(RSATB_NUMERICAL_FAILURE, "lanczos: non-finite coefficient at step %d", j);
        alpha[j] = a;
        beta[j] = b;
        if (b < 1e-12 * std::max(1.0, std::fabs(a))) {  // invariant subspace
            used = j + 1;
            converged = true;
            break;
        }
        if (converge && j >= 3 && j % 2 == 1) {
            RSATB_TRY(tridiag_eigen(j + 1, alpha.data(), beta.data(), th.data(), yl.data()));
            const double scale = std::max({std::fabs(th[0]), std::fabs(th[j]), 1e-300});
            if (std::fabs(b * yl[0]) <= o.tol * scale && std::fabs(b * yl[j]) <= o.tol * scale) {
                used = j + 1;
                converged = true;
                break;
            }
        }
        if (j + 1 < m) {
            scale_copy<<<eg, 256, 0, st>>>(w, 1.0 / b, vals, Q + int64_t(j + 1) * ld);
            RSATB_LAUNCH_CHECK(ctx);
        }
    }
    RSATB_TRY(tridiag_eigen(used, alpha.data(), beta.data(), th.data(), yl.data()));
    result->theta_min = th[0];
    result->theta_max = th[used - 1];
    result->res_min = std::fabs(beta[used - 1] * yl[0]);
    result->res_max = std::fabs(beta[used - 1] * yl[used - 1]);
    result->matvecs = used;
    result->converged = converged ? 1 : 0;
    RSATB_CUDA_TRY(cudaStreamSynchronize(st));
    return ctx_check_fault(ctx);
}
