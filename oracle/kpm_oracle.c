/*
 * kpm_oracle.c -- TEST INFRASTRUCTURE.  CPU restatement, in plain C with
 * OpenMP, of the reference algorithms on the KPM / transport hot path.  It
 * is the checker the GPU library is compared against (and the timed CPU
 * baseline of bench.py); nothing in the product calls it.
 *
 * Every routine follows a reference function, cited at its definition.
 * Arithmetic is FP64 throughout (the reference Scalar is complex<double>,
 * rsatb/rsatb.hpp:53).  Parallel reductions use a static row partition
 * and combine the per-thread sums in thread order, so results are
 * reproducible for a fixed thread count.
 *
 * Conventions (identical to include/rsatb_b200.h):
 *   multivector  N x W reals row-major; a complex multivector of R columns
 *                has W = 2R with (re, im) interleaved.
 *   BSR          uniform b x b blocks, row-major values, complex interleaved;
 *                `imag` marks a real-valued matrix that stands for i*W.
 *   <a|b>        sum_i conj(a_i) b_i per column.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int n_block_rows;
    int n_block_cols;
    int b;
    const int32_t* row_ptr;
    const int32_t* col_ind;
    const double* vals;
    int cplx; /* complex values */
    int imag; /* real values standing for i * values */
} orc_bsr;

static int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int orc_num_threads(void) { return orc_threads(); }

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------ Philox */

/* Philox-4x32-10 (Salmon et al., SC'11): ten rounds of two 32x32->64
 * multiplications with Weyl-sequence key increments. */
static void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)M0 * c[0];
        const uint64_t p1 = (uint64_t)M1 * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c[1] ^ k0;
        const uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += W0;
        k1 += W1;
    }
}

static const double SIN_C[12] = {-0.16666666666666666,    0.008333333333333333,
                                 -0.0001984126984126984,  2.7557319223985893e-06,
                                 -2.505210838544172e-08,  1.6059043836821613e-10,
                                 -7.647163731819816e-13,  2.8114572543455206e-15,
                                 -8.22063524662433e-18,   1.9572941063391263e-20,
                                 -3.868170170630684e-23,  6.446950284384474e-26};
static const double COS_C[13] = {-0.5,
                                 0.041666666666666664,
                                 -0.001388888888888889,
                                 2.48015873015873e-05,
                                 -2.755731922398589e-07,
                                 2.08767569878681e-09,
                                 -1.1470745597729725e-11,
                                 4.779477332387385e-14,
                                 -1.5619206968586225e-16,
                                 4.110317623312165e-19,
                                 -8.896791392450574e-22,
                                 1.6117375710961184e-24,
                                 -2.4795962632247976e-27};

/* cos and sin of 2 pi u53 / 2^53 by quadrant reduction and Taylor series
 * (explicit fma, no libm), the sample-vector phase definition. */
static void phase_of(uint64_t u53, double* co, double* si) {
    const unsigned quad = (unsigned)(u53 >> 51);
    const uint64_t f = u53 & ((((uint64_t)1) << 51) - 1);
    volatile double t = (double)f * 4.440892098500626e-16;
    int fold = t > 0.5;
    double tt = fold ? 1.0 - t : t;
    volatile double psi = tt * 1.5707963267948966;
    volatile double z = psi * psi;
    double ps = SIN_C[11];
    for (int k = 10; k >= 0; --k) ps = fma(ps, z, SIN_C[k]);
    volatile double pz = psi * z;
    const double s = fma(pz, ps, psi);
    double pc = COS_C[12];
    for (int k = 11; k >= 0; --k) pc = fma(pc, z, COS_C[k]);
    const double c = fma(z, pc, 1.0);
    const double cq = fold ? s : c, sq = fold ? c : s;
    switch (quad) {
        case 0: *co = cq; *si = sq; break;
        case 1: *co = -sq; *si = cq; break;
        case 2: *co = -cq; *si = -sq; break;
        default: *co = sq; *si = -cq; break;
    }
}

/* Sample vectors (rsatb/calc/observables.hpp:84-96, vbcsr set_random):
 * element (row, col) from (seed, atom_index[atom], orbital, col).
 * kind 0 phase, 1 Rademacher, 2 uniform [-1, 1).  out is N x W. */
int orc_set_random(uint64_t seed, int kind, int normalize, const int64_t* atom_index, int n_atoms,
                   int orbitals, int64_t n_rows_global, int n_vectors, int64_t first_column,
                   int complex_out, double* out) {
    if (kind == 0 && !complex_out) return 1;
    const double scale = normalize ? 1.0 / sqrt((double)n_rows_global) : 1.0;
    const int64_t n_rows = (int64_t)n_atoms * orbitals;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma omp parallel for schedule(static)
    for (int64_t row = 0; row < n_rows; ++row) {
        const int64_t atom = row / orbitals;
        const int orb = (int)(row - atom * orbitals);
        const uint64_t id = (uint64_t)atom_index[atom];
        for (int col = 0; col < n_vectors; ++col) {
            uint32_t c[4] = {(uint32_t)id, (uint32_t)(id >> 32), (uint32_t)orb,
                             (uint32_t)(first_column + col)};
            philox(c, k0, k1);
            double re = 0.0, im = 0.0;
            if (kind == 0) {
                const uint64_t u53 = ((uint64_t)c[0] << 21) ^ (uint64_t)(c[1] >> 11);
                phase_of(u53, &re, &im);
                volatile double a = re * scale, b = im * scale;
                re = a;
                im = b;
            } else if (kind == 1) {
                re = (c[2] & 1u) ? -scale : scale;
            } else {
                const uint64_t a = ((uint64_t)c[0] << 21) ^ (uint64_t)(c[1] >> 11);
                const uint64_t b = ((uint64_t)c[2] << 21) ^ (uint64_t)(c[3] >> 11);
                volatile double ra = (double)((int64_t)(2 * a) - ((int64_t)1 << 53)) *
                                     1.1102230246251565e-16;
                volatile double rb = (double)((int64_t)(2 * b) - ((int64_t)1 << 53)) *
                                     1.1102230246251565e-16;
                volatile double sa = ra * scale, sb = rb * scale;
                re = sa;
                im = sb;
            }
            const int64_t e = row * n_vectors + col;
            if (complex_out) {
                out[2 * e] = re;
                out[2 * e + 1] = im;
            } else {
                out[e] = re;
            }
        }
    }
    return 0;
}

/* -------------------------------------------------------------- BSR SpMM */

/* Y = alpha * A X (vbcsr BlockSpMat::mult_dense, the only matrix kernel
 * Chebyshev::mult_by calls, rsatb/calc/cheby.hpp:599-606).  cv: X and Y are
 * complex panels (W = 2R). */
void orc_spmm(const orc_bsr* A, const double* X, double* Y, int W, int cv, double alpha) {
    const int b = A->b;
    const int64_t bb = (int64_t)b * b;
#pragma omp parallel
    {
        double* acc = (double*)malloc(sizeof(double) * (size_t)W);
#pragma omp for schedule(static)
        for (int i = 0; i < A->n_block_rows; ++i) {
            for (int r = 0; r < b; ++r) {
                for (int w = 0; w < W; ++w) acc[w] = 0.0;
                for (int k = A->row_ptr[i]; k < A->row_ptr[i + 1]; ++k) {
                    const int64_t j = A->col_ind[k];
                    for (int c = 0; c < b; ++c) {
                        const double* x = X + (j * b + c) * W;
                        if (A->cplx) {
                            const double ar = A->vals[2 * (k * bb + r * b + c)];
                            const double ai = A->vals[2 * (k * bb + r * b + c) + 1];
                            for (int w = 0; w < W; w += 2) {
                                acc[w] += ar * x[w] - ai * x[w + 1];
                                acc[w + 1] += ar * x[w + 1] + ai * x[w];
                            }
                        } else {
                            const double a = A->vals[k * bb + r * b + c];
                            for (int w = 0; w < W; ++w) acc[w] += a * x[w];
                        }
                    }
                }
                double* y = Y + ((int64_t)i * b + r) * W;
                if (A->imag) {
                    for (int w = 0; w < W; w += 2) {
                        y[w] = -acc[w + 1] * alpha;
                        y[w + 1] = acc[w] * alpha;
                    }
                } else {
                    for (int w = 0; w < W; ++w) y[w] = acc[w] * alpha;
                }
            }
        }
        free(acc);
    }
    (void)cv;
}

/* Per-column <a|b> over n rows into out[W] (complex: (re, im) pairs). */
static void coldots(const double* a, const double* b, int64_t n, int W, int cv, double* out) {
    const int nt = orc_threads();
    double* part = (double*)calloc((size_t)nt * W, sizeof(double));
#pragma omp parallel
    {
#ifdef _OPENMP
        const int tid = omp_get_thread_num();
#else
        const int tid = 0;
#endif
        double* p = part + (size_t)tid * W;
#pragma omp for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            const double* x = a + i * W;
            const double* y = b + i * W;
            if (cv) {
                for (int w = 0; w < W; w += 2) {
                    p[w] += x[w] * y[w] + x[w + 1] * y[w + 1];
                    p[w + 1] += x[w] * y[w + 1] - x[w + 1] * y[w];
                }
            } else {
                for (int w = 0; w < W; ++w) p[w] += x[w] * y[w];
            }
        }
    }
    for (int w = 0; w < W; ++w) {
        double s = 0.0;
        for (int t = 0; t < nt; ++t) s += part[(size_t)t * W + w];
        out[w] = s;
    }
    free(part);
}

/* y = a*x + b*y (DistMultiVector::axpby). */
static void axpby(double a, const double* x, double b, double* y, int64_t n) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) y[i] = a * x[i] + b * y[i];
}

/* -------------------------------------------------- the rescaled operator */

typedef struct {
    int sandwich;
    const orc_bsr* H;
    const orc_bsr* Z;
    const orc_bsr* ZH;
    double center;
    double half_width;
} orc_op;

/* y = ((Op) x - c x)/hw, Chebyshev::apply_form (rsatb/calc/cheby.hpp:
 * 555-591) in its order: the operator, then y.axpy(-center, x), then
 * y.scale(1/half_width).  Sandwich: y = Z^H (H (Z x)) with scratch t. */
void orc_apply_op(const orc_op* op, const double* x, double* y, int W, int cv, double* t) {
    const int64_t N = (int64_t)op->H->n_block_rows * op->H->b;
    if (op->sandwich) {
        orc_spmm(op->Z, x, y, W, cv, 1.0);    /* y = Z x */
        orc_spmm(op->H, y, t, W, cv, 1.0);    /* t = H Z x */
        orc_spmm(op->ZH, t, y, W, cv, 1.0);   /* y = Z^H H Z x */
    } else {
        orc_spmm(op->H, x, y, W, cv, 1.0);
    }
    const int64_t n = N * W;
    const double c = op->center, s = 1.0 / op->half_width;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        y[i] = y[i] + (-c) * x[i];
        y[i] = y[i] * s;
    }
}

/* ----------------------------------------------------------- KPM moments */

/* rsatb::calc::kpm_dos_moments, multivector overload (rsatb/calc/dos.hpp:
 * 125-190): doubled when `doubled` (op Hermitian), plain otherwise.  The
 * per-column dots are averaged over columns (dos.hpp:134-138) before the
 * doubling formulas.  mu_out: 2*n_moments doubles (complex).  col_mu (may be
 * NULL): per-column moments [n_moments][R] complex, the doubling formula
 * applied column by column. */
int orc_kpm_moments(const orc_op* op, const double* psi, int R, int cv, int n_moments, int doubled,
                    double* mu_out, double* col_mu) {
    const int W = cv ? 2 * R : R;
    const int64_t N = (int64_t)op->H->n_block_rows * op->H->b;
    const int64_t n = N * W;
    double* t0 = (double*)malloc(sizeof(double) * (size_t)n);
    double* t1 = (double*)malloc(sizeof(double) * (size_t)n);
    double* t2 = (double*)malloc(sizeof(double) * (size_t)n);
    double* tmp = (double*)malloc(sizeof(double) * (size_t)n);
    double* d = (double*)malloc(sizeof(double) * (size_t)W);
    double* cm = (double*)calloc((size_t)n_moments * 2 * R, sizeof(double));
    if (!t0 || !t1 || !t2 || !tmp || !d || !cm) return 2;
    for (int i = 0; i < 2 * n_moments; ++i) mu_out[i] = 0.0;
    memcpy(t0, psi, sizeof(double) * (size_t)n);

    /* averaged(): sum of per-column complex dots / num_vecs */
#define COLRE(q) (cv ? d[2 * (q)] : d[(q)])
#define COLIM(q) (cv ? d[2 * (q) + 1] : 0.0)
#define AVERAGE(re_, im_)                                   \
    do {                                                    \
        double sr_ = 0.0, si_ = 0.0;                        \
        for (int q_ = 0; q_ < R; ++q_) {                    \
            sr_ += COLRE(q_);                               \
            si_ += COLIM(q_);                               \
        }                                                   \
        re_ = sr_ / (double)R;                              \
        im_ = si_ / (double)R;                              \
    } while (0)
#define SETCOL(m, q, re_, im_)                              \
    do {                                                    \
        cm[2 * ((size_t)(m) * R + (q))] = (re_);            \
        cm[2 * ((size_t)(m) * R + (q)) + 1] = (im_);        \
    } while (0)

    coldots(t0, t0, N, W, cv, d);
    double mu0r, mu0i;
    AVERAGE(mu0r, mu0i);
    mu_out[0] = mu0r;
    mu_out[1] = mu0i;
    for (int q = 0; q < R; ++q) SETCOL(0, q, COLRE(q), COLIM(q));
    double* colmu0 = (double*)malloc(sizeof(double) * 2 * R);
    double* colmu1 = (double*)malloc(sizeof(double) * 2 * R);
    for (int q = 0; q < R; ++q) {
        colmu0[2 * q] = COLRE(q);
        colmu0[2 * q + 1] = COLIM(q);
    }
    if (n_moments > 1) {
        orc_apply_op(op, t0, t1, W, cv, tmp);
        coldots(t0, t1, N, W, cv, d);  /* t0.dot(t1) */
        double r, i;
        AVERAGE(r, i);
        mu_out[2] = r;
        mu_out[3] = i;
        for (int q = 0; q < R; ++q) {
            SETCOL(1, q, COLRE(q), COLIM(q));
            colmu1[2 * q] = COLRE(q);
            colmu1[2 * q + 1] = COLIM(q);
        }
        if (doubled) {
            for (int k = 1;; ++k) {
                if (2 * k - 1 < n_moments && 2 * k - 1 > 1) {
                    coldots(t1, t0, N, W, cv, d);
                    AVERAGE(r, i);
                    mu_out[2 * (2 * k - 1)] = 2.0 * r - mu_out[2];
                    mu_out[2 * (2 * k - 1) + 1] = 2.0 * i - mu_out[3];
                    for (int q = 0; q < R; ++q)
                        SETCOL(2 * k - 1, q, 2.0 * COLRE(q) - colmu1[2 * q],
                               2.0 * COLIM(q) - colmu1[2 * q + 1]);
                }
                if (2 * k < n_moments) {
                    coldots(t1, t1, N, W, cv, d);
                    AVERAGE(r, i);
                    mu_out[2 * (2 * k)] = 2.0 * r - mu_out[0];
                    mu_out[2 * (2 * k) + 1] = 2.0 * i - mu_out[1];
                    for (int q = 0; q < R; ++q)
                        SETCOL(2 * k, q, 2.0 * COLRE(q) - colmu0[2 * q],
                               2.0 * COLIM(q) - colmu0[2 * q + 1]);
                }
                if (2 * k + 1 >= n_moments) break;
                orc_apply_op(op, t1, t2, W, cv, tmp);
                axpby(-1.0, t0, 2.0, t2, n);
                double* s = t0;
                t0 = t1;
                t1 = t2;
                t2 = s;
            }
        } else {
            for (int k = 2; k < n_moments; ++k) {
                orc_apply_op(op, t1, t2, W, cv, tmp);
                axpby(-1.0, t0, 2.0, t2, n);
                coldots(psi, t2, N, W, cv, d);
                AVERAGE(r, i);
                mu_out[2 * k] = r;
                mu_out[2 * k + 1] = i;
                for (int q = 0; q < R; ++q) SETCOL(k, q, COLRE(q), COLIM(q));
                double* s = t0;
                t0 = t1;
                t1 = t2;
                t2 = s;
            }
        }
    }
    if (col_mu) memcpy(col_mu, cm, sizeof(double) * (size_t)n_moments * 2 * R);
#undef COLRE
#undef COLIM
#undef AVERAGE
#undef SETCOL
    free(colmu0);
    free(colmu1);
    free(t0);
    free(t1);
    free(t2);
    free(tmp);
    free(d);
    free(cm);
    return 0;
}

/* --------------------------------------------------- kernels and density */

/* kpm_kernel_weights (rsatb/calc/kpm.hpp:52-85); jackson_kernel :18-26.
 * kernel: 0 none, 1 Jackson, 2 CosTaper, 3 VpTaper. */
void orc_kernel_weights(int kernel, int n, double* g) {
    for (int i = 0; i < n; ++i) g[i] = 1.0;
    if (kernel == 1) {
        const double denom = (double)(n + 1);
        const double theta = M_PI / denom;
        const double cot_theta = cos(theta) / sin(theta);
        g[0] = 1.0;
        for (int i = 1; i < n; ++i)
            g[i] = ((denom - i) * cos(theta * i) + cot_theta * sin(theta * i)) / denom;
    } else if (kernel == 2) {
        const int n0 = n / 2;
        for (int i = n0; i < n; ++i) {
            const double s = (double)(i - n0) / (double)(n - n0);
            g[i] = 0.5 * (1.0 + cos(M_PI * s));
        }
    } else if (kernel == 3) {
        const int n0 = n / 2;
        for (int i = n0; i < n; ++i) g[i] = (double)(n - i) / (double)(n - n0);
    }
}

/* evaluate_kpm_density (rsatb/calc/kpm.hpp:206-241); moments complex
 * (2*n doubles), real parts used. */
void orc_density(const double* mu, int n, const double* x, int nx, double edge_inset, int kernel,
                 double* rho) {
    double* g = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    orc_kernel_weights(kernel, n, g);
    for (int j = 0; j < nx; ++j) {
        if (n == 0) {
            rho[j] = 0.0;
            continue;
        }
        double xj = x[j];
        if (xj > 1.0 - edge_inset) xj = 1.0 - edge_inset;
        if (xj < -1.0 + edge_inset) xj = -1.0 + edge_inset;
        double t_prev = 1.0, t_curr = xj;
        double acc = g[0] * mu[0];
        if (n > 1) acc += 2.0 * g[1] * mu[2] * t_curr;
        for (int k = 2; k < n; ++k) {
            const double t_next = 2.0 * xj * t_curr - t_prev;
            acc += 2.0 * g[k] * mu[2 * k] * t_next;
            t_prev = t_curr;
            t_curr = t_next;
        }
        const double w = 1.0 - xj * xj;
        rho[j] = acc / (M_PI * sqrt(w > 1e-14 ? w : 1e-14));
    }
    free(g);
}

/* ------------------------------------------------------------- DCT-III */

/* y_k = x_0 + 2 sum_{m>=1} x_m cos(pi m (k + 1/2) / n), complex x, by the
 * explicit cosine sum (the check in test_fftcheb_transport.cpp:476-545). */
void orc_dct3_direct(const double* in, int n, int batch, double* out) {
#pragma omp parallel for schedule(static)
    for (int b = 0; b < batch; ++b) {
        const double* x = in + (size_t)b * 2 * n;
        double* y = out + (size_t)b * 2 * n;
        for (int k = 0; k < n; ++k) {
            double re = x[0], im = x[1];
            for (int m = 1; m < n; ++m) {
                const double c = cos(M_PI * (double)m * ((double)k + 0.5) / (double)n);
                re += 2.0 * x[2 * m] * c;
                im += 2.0 * x[2 * m + 1] * c;
            }
            y[2 * k] = re;
            y[2 * k + 1] = im;
        }
    }
}

/* The RowFFTWorkspace::dct_type3_batch route (rsatb/calc/fft.hpp:125-154):
 * even extension with the half-grid phase e^{+-i pi m / 2n}, then the
 * unnormalised inverse 2n-point DFT, first n outputs kept.  The DFT is
 * evaluated directly (oracle sizes are small). */
void orc_dct3_fftroute(const double* in, int n, int batch, double* out) {
    const int nn = 2 * n;
#pragma omp parallel
    {
        double* e = (double*)malloc(sizeof(double) * 2 * (size_t)nn);
#pragma omp for schedule(static)
        for (int b = 0; b < batch; ++b) {
            const double* x = in + (size_t)b * 2 * n;
            for (int i = 0; i < 2 * nn; ++i) e[i] = 0.0;
            e[0] = x[0];
            e[1] = x[1];
            for (int m = 1; m < n; ++m) {
                const double th = M_PI * (double)m / (2.0 * (double)n);
                const double c = cos(th), s = sin(th);
                const double vr = x[2 * m], vi = x[2 * m + 1];
                e[2 * m] = vr * c - vi * s;
                e[2 * m + 1] = vr * s + vi * c;
                e[2 * (nn - m)] = vr * c + vi * s;
                e[2 * (nn - m) + 1] = -vr * s + vi * c;
            }
            double* y = out + (size_t)b * 2 * n;
            for (int k = 0; k < n; ++k) {
                double re = 0.0, im = 0.0;
                for (int j = 0; j < nn; ++j) {
                    const double ang = 2.0 * M_PI * (double)((int64_t)j * k % nn) / (double)nn;
                    const double c = cos(ang), s = sin(ang);
                    re += e[2 * j] * c - e[2 * j + 1] * s;
                    im += e[2 * j] * s + e[2 * j + 1] * c;
                }
                y[2 * k] = re;
                y[2 * k + 1] = im;
            }
        }
        free(e);
    }
}

/* ------------------------------------------------ FFT-Chebyshev transport */

/* Unnormalised inverse DFT (sign +) of length n over interleaved complex;
 * iterative radix-2 when n is a power of two, direct sum otherwise. */
static void idft(double* a, int n, double* work) {
    if (n > 1 && (n & (n - 1)) == 0) {
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) {
                double t0 = a[2 * i], t1 = a[2 * i + 1];
                a[2 * i] = a[2 * j];
                a[2 * i + 1] = a[2 * j + 1];
                a[2 * j] = t0;
                a[2 * j + 1] = t1;
            }
        }
        for (int len = 2; len <= n; len <<= 1) {
            const double ang = 2.0 * M_PI / (double)len;
            for (int i = 0; i < n; i += len) {
                for (int k = 0; k < len / 2; ++k) {
                    const double wr = cos(ang * k), wi = sin(ang * k);
                    double* u = a + 2 * (i + k);
                    double* v = a + 2 * (i + k + len / 2);
                    const double vr = v[0] * wr - v[1] * wi, vi = v[0] * wi + v[1] * wr;
                    v[0] = u[0] - vr;
                    v[1] = u[1] - vi;
                    u[0] += vr;
                    u[1] += vi;
                }
            }
        }
        return;
    }
    for (int k = 0; k < n; ++k) {
        double re = 0.0, im = 0.0;
        for (int j = 0; j < n; ++j) {
            const double ang = 2.0 * M_PI * (double)((int64_t)j * k % n) / (double)n;
            const double c = cos(ang), s = sin(ang);
            re += a[2 * j] * c - a[2 * j + 1] * s;
            im += a[2 * j] * s + a[2 * j + 1] * c;
        }
        work[2 * k] = re;
        work[2 * k + 1] = im;
    }
    memcpy(a, work, sizeof(double) * 2 * (size_t)n);
}

/* dct_type3 of one complex sequence of length n (fft.hpp:125-154). */
static void dct3_one(const double* x, int n, double* y, double* e, double* work) {
    const int nn = 2 * n;
    for (int i = 0; i < 2 * nn; ++i) e[i] = 0.0;
    e[0] = x[0];
    e[1] = x[1];
    for (int m = 1; m < n; ++m) {
        const double th = M_PI * (double)m / (2.0 * (double)n);
        const double c = cos(th), s = sin(th);
        const double vr = x[2 * m], vi = x[2 * m + 1];
        e[2 * m] = vr * c - vi * s;
        e[2 * m + 1] = vr * s + vi * c;
        e[2 * (nn - m)] = vr * c + vi * s;
        e[2 * (nn - m) + 1] = -vr * s + vi * c;
    }
    idft(e, nn, work);
    memcpy(y, e, sizeof(double) * 2 * (size_t)n);
}

/* zero_padded_ifft of one sequence (fft.hpp:156-174): inverse 2n DFT of x
 * padded with zeros, first n outputs. */
static void zpifft_one(const double* x, int n, double* y, double* e, double* work) {
    const int nn = 2 * n;
    for (int i = 0; i < 2 * nn; ++i) e[i] = 0.0;
    memcpy(e, x, sizeof(double) * 2 * (size_t)n);
    idft(e, nn, work);
    memcpy(y, e, sizeof(double) * 2 * (size_t)n);
}

static int comp_index(int a, int b) {
    if (a > b) {
        int t = a;
        a = b;
        b = t;
    }
    return (-a * a + 5 * a) / 2 + b;
}

/* y = scale * (dressed V) x: Chebyshev::apply_dual for a bare matrix
 * (rsatb/calc/cheby.hpp:249-291): V x (Orthogonal) or Z^H V Z x (Sandwich),
 * then y.scale(scale).  NORMAL and ADJOINT agree for these two forms. */
static void apply_dual(const orc_op* op, const orc_bsr* V, const double* x, double* y, int W,
                       double scale, double* t) {
    const int64_t n = (int64_t)op->H->n_block_rows * op->H->b * W;
    if (op->sandwich) {
        orc_spmm(op->Z, x, y, W, 1, 1.0);
        orc_spmm(V, y, t, W, 1, 1.0);
        orc_spmm(op->ZH, t, y, W, 1, 1.0);
    } else {
        orc_spmm(V, x, y, W, 1, 1.0);
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) y[i] = y[i] * scale;
}

/* store_axis_rows (fftcheb_transport.hpp:234-258) into the
 * [row][axis][sample][moment] layout of fftcheb_store_offset (:145-156). */
static void store_rows(const double* vec, double* store, int row_begin, int row_count, int axis,
                       int m, int R, int M) {
    for (int r = 0; r < row_count; ++r)
        for (int s = 0; s < R; ++s) {
            const size_t off = ((((size_t)r * 3 + axis) * R + s) * M + m);
            store[2 * off] = vec[2 * ((size_t)(row_begin + r) * R + s)];
            store[2 * off + 1] = vec[2 * ((size_t)(row_begin + r) * R + s) + 1];
        }
}

/* dc_spectrum_fftcheb (rsatb/calc/fftcheb_transport.hpp:543-660) with one
 * sample block of all R samples, driving accumulate_fftcheb_block
 * (:270-525).  formulation 0 Greenwood, 1 Bastin.  psi: N x R complex.
 * sigma_out: n_moments*6, energy_out: n_moments, ascending. */
int orc_fftcheb(const orc_op* op, const orc_bsr* Vx, const orc_bsr* Vy, const orc_bsr* Vz,
                const double* psi, int R, int M, int formulation, double prefactor,
                int sections, int kernel, double* sigma_out, double* energy_out) {
    const orc_bsr* V[3] = {Vx, Vy, Vz};
    const int N = op->H->n_block_rows * op->H->b;
    const int W = 2 * R;
    const size_t nv = (size_t)N * W;
    double* g = (double*)malloc(sizeof(double) * M);
    orc_kernel_weights(kernel, M, g);
    double* phi3w = (double*)malloc(sizeof(double) * M);
    double* pw = (double*)malloc(sizeof(double) * 2 * M);   /* phase_weight */
    double* pwm = (double*)malloc(sizeof(double) * 2 * M);  /* phase_weight_m */
    double* eps = (double*)malloc(sizeof(double) * M);
    double* root = (double*)malloc(sizeof(double) * M);
    for (int m = 0; m < M; ++m) {
        const double coeff = 2.0 * g[m] / (M_PI * (1.0 + (m == 0 ? 1.0 : 0.0)));
        phi3w[m] = g[m] / M_PI;
        const double th = M_PI * (double)m / (2.0 * (double)M);
        pw[2 * m] = coeff * cos(th);
        pw[2 * m + 1] = coeff * sin(th);
        pwm[2 * m] = pw[2 * m] * (double)m;
        pwm[2 * m + 1] = pw[2 * m + 1] * (double)m;
    }
    for (int k = 0; k < M; ++k) {
        const double th = M_PI * ((double)k + 0.5) / (double)M;
        eps[k] = cos(th);
        root[k] = sin(th);
    }
    const double vscale = 1.0 / (2.0 * op->half_width);
    double* K = (double*)calloc((size_t)M * 6 * 2, sizeof(double));

    double *rinit[3], *rprev[3], *rcurr[3], *rnext[3], *laxes[3];
    for (int a = 0; a < 3; ++a) {
        rinit[a] = (double*)malloc(sizeof(double) * nv);
        rprev[a] = (double*)malloc(sizeof(double) * nv);
        rcurr[a] = (double*)malloc(sizeof(double) * nv);
        rnext[a] = (double*)malloc(sizeof(double) * nv);
        laxes[a] = (double*)malloc(sizeof(double) * nv);
    }
    double* lprev = (double*)malloc(sizeof(double) * nv);
    double* lcurr = (double*)malloc(sizeof(double) * nv);
    double* lnext = (double*)malloc(sizeof(double) * nv);
    double* tmp = (double*)malloc(sizeof(double) * nv);
    for (int a = 0; a < 3; ++a) apply_dual(op, V[a], psi, rinit[a], W, -vscale, tmp);

    const int n_sections = sections > 0 ? sections : 1;
    const int section_rows = (N + n_sections - 1) / n_sections > 0 ? (N + n_sections - 1) / n_sections : 1;
    for (int sec = 0; sec < n_sections; ++sec) {
        const int row_begin = sec * section_rows;
        const int row_end = row_begin + section_rows < N ? row_begin + section_rows : N;
        const int rc = row_end - row_begin;
        if (rc <= 0) continue;
        const size_t store_n = (size_t)rc * 3 * R * M;
        double* lstore = (double*)calloc(2 * store_n, sizeof(double));
        double* rstore = (double*)calloc(2 * store_n, sizeof(double));
        for (int a = 0; a < 3; ++a) memcpy(rprev[a], rinit[a], sizeof(double) * nv);
        memcpy(lprev, psi, sizeof(double) * nv);
        for (int a = 0; a < 3; ++a) apply_dual(op, V[a], lprev, laxes[a], W, -vscale, tmp);
        for (int a = 0; a < 3; ++a) {
            store_rows(laxes[a], lstore, row_begin, rc, a, 0, R, M);
            store_rows(rprev[a], rstore, row_begin, rc, a, 0, R, M);
        }
        if (M > 1) {
            for (int a = 0; a < 3; ++a) orc_apply_op(op, rprev[a], rcurr[a], W, 1, tmp);
            orc_apply_op(op, lprev, lcurr, W, 1, tmp);
            for (int a = 0; a < 3; ++a) apply_dual(op, V[a], lcurr, laxes[a], W, -vscale, tmp);
            for (int a = 0; a < 3; ++a) {
                store_rows(laxes[a], lstore, row_begin, rc, a, 1, R, M);
                store_rows(rcurr[a], rstore, row_begin, rc, a, 1, R, M);
            }
        }
        for (int m = 2; m < M; ++m) {
            for (int a = 0; a < 3; ++a) {
                orc_apply_op(op, rcurr[a], rnext[a], W, 1, tmp);
                axpby(-1.0, rprev[a], 2.0, rnext[a], (int64_t)nv);
            }
            orc_apply_op(op, lcurr, lnext, W, 1, tmp);
            axpby(-1.0, lprev, 2.0, lnext, (int64_t)nv);
            for (int a = 0; a < 3; ++a) apply_dual(op, V[a], lnext, laxes[a], W, -vscale, tmp);
            for (int a = 0; a < 3; ++a) {
                store_rows(laxes[a], lstore, row_begin, rc, a, m, R, M);
                store_rows(rnext[a], rstore, row_begin, rc, a, m, R, M);
                double* s = rprev[a];
                rprev[a] = rcurr[a];
                rcurr[a] = rnext[a];
                rnext[a] = s;
            }
            double* s = lprev;
            lprev = lcurr;
            lcurr = lnext;
            lnext = s;
        }
        /* Row stage: per-row transforms and the rowwise contraction. */
        const int nt = orc_threads();
        double* Kpart = (double*)calloc((size_t)nt * M * 6 * 2, sizeof(double));
#pragma omp parallel
        {
#ifdef _OPENMP
            const int tid = omp_get_thread_num();
#else
            const int tid = 0;
#endif
            double* Kp = Kpart + (size_t)tid * M * 12;
            const size_t seqn = (size_t)R * M * 2;
            double* wbuf = (double*)malloc(sizeof(double) * 2 * M);
            double* e = (double*)malloc(sizeof(double) * 4 * M);
            double* work = (double*)malloc(sizeof(double) * 4 * M);
            double* L3 = (double*)malloc(sizeof(double) * 3 * seqn);
            double* R3 = (double*)malloc(sizeof(double) * 3 * seqn);
            double* L1 = (double*)malloc(sizeof(double) * 3 * seqn);
            double* L2 = (double*)malloc(sizeof(double) * 3 * seqn);
            double* R1 = (double*)malloc(sizeof(double) * 3 * seqn);
            double* R2 = (double*)malloc(sizeof(double) * 3 * seqn);
#pragma omp for schedule(static)
            for (int row = 0; row < rc; ++row) {
                for (int a = 0; a < 3; ++a) {
                    const double* lrow = lstore + 2 * (((size_t)row * 3 + a) * R * M);
                    const double* rrow = rstore + 2 * (((size_t)row * 3 + a) * R * M);
                    for (int s = 0; s < R; ++s) {
                        const double* ls = lrow + 2 * (size_t)s * M;
                        const double* rs = rrow + 2 * (size_t)s * M;
                        double* l3 = L3 + a * seqn + 2 * (size_t)s * M;
                        double* r3 = R3 + a * seqn + 2 * (size_t)s * M;
                        for (int m = 0; m < M; ++m) {
                            wbuf[2 * m] = phi3w[m] * ls[2 * m];
                            wbuf[2 * m + 1] = phi3w[m] * ls[2 * m + 1];
                        }
                        dct3_one(wbuf, M, l3, e, work);
                        for (int m = 0; m < M; ++m) {
                            wbuf[2 * m] = phi3w[m] * rs[2 * m];
                            wbuf[2 * m + 1] = phi3w[m] * rs[2 * m + 1];
                        }
                        dct3_one(wbuf, M, r3, e, work);
                        if (formulation == 1) {
                            const double* ws[2] = {pw, pwm};
                            double* lo[2] = {L1 + a * seqn + 2 * (size_t)s * M,
                                             L2 + a * seqn + 2 * (size_t)s * M};
                            double* ro[2] = {R1 + a * seqn + 2 * (size_t)s * M,
                                             R2 + a * seqn + 2 * (size_t)s * M};
                            for (int q = 0; q < 2; ++q) {
                                for (int m = 0; m < M; ++m) {
                                    wbuf[2 * m] = ws[q][2 * m] * ls[2 * m] - ws[q][2 * m + 1] * ls[2 * m + 1];
                                    wbuf[2 * m + 1] = ws[q][2 * m] * ls[2 * m + 1] + ws[q][2 * m + 1] * ls[2 * m];
                                }
                                zpifft_one(wbuf, M, lo[q], e, work);
                                for (int m = 0; m < M; ++m) {
                                    wbuf[2 * m] = ws[q][2 * m] * rs[2 * m] - ws[q][2 * m + 1] * rs[2 * m + 1];
                                    wbuf[2 * m + 1] = ws[q][2 * m] * rs[2 * m + 1] + ws[q][2 * m + 1] * rs[2 * m];
                                }
                                zpifft_one(wbuf, M, ro[q], e, work);
                            }
                        }
                    }
                }
                if (formulation == 0) {
                    for (int a = 0; a < 3; ++a) {
                        const int comp = comp_index(a, a);
                        for (int k = 0; k < M; ++k) {
                            const double w = 1.0 - eps[k] * eps[k];
                            const double denom = w > 1e-14 ? w : 1e-14;
                            double ar = 0.0, ai = 0.0;
                            for (int s = 0; s < R; ++s) {
                                const double* l = L3 + a * seqn + 2 * ((size_t)s * M + k);
                                const double* r = R3 + a * seqn + 2 * ((size_t)s * M + k);
                                ar += l[0] * r[0] + l[1] * r[1];
                                ai += l[0] * r[1] - l[1] * r[0];
                            }
                            Kp[2 * (k * 6 + comp)] += ar / denom;
                            Kp[2 * (k * 6 + comp) + 1] += ai / denom;
                        }
                    }
                } else {
                    for (int a = 0; a < 3; ++a)
                        for (int b2 = a; b2 < 3; ++b2) {
                            const int comp = comp_index(a, b2);
                            for (int k = 0; k < M; ++k) {
                                double vr = 0.0, vi = 0.0;
                                for (int s = 0; s < R; ++s) {
                                    const size_t i = 2 * ((size_t)s * M + k);
                                    const double* l3 = L3 + a * seqn + i;
                                    const double* l1 = L1 + a * seqn + i;
                                    const double* l2 = L2 + a * seqn + i;
                                    const double* r3 = R3 + b2 * seqn + i;
                                    const double* r1 = R1 + b2 * seqn + i;
                                    const double* r2 = R2 + b2 * seqn + i;
                                    /* conj(x) y */
#define CJR(x, y) ((x)[0] * (y)[0] + (x)[1] * (y)[1])
#define CJI(x, y) ((x)[0] * (y)[1] - (x)[1] * (y)[0])
                                    const double tr = CJR(l3, r1) + CJR(l1, r3);
                                    const double ti = CJI(l3, r1) + CJI(l1, r3);
                                    const double ur = CJR(l2, r3) - CJR(l3, r2);
                                    const double ui = CJI(l2, r3) - CJI(l3, r2);
#undef CJR
#undef CJI
                                    /* eps*t + i*root*u */
                                    vr += eps[k] * tr - root[k] * ui;
                                    vi += eps[k] * ti + root[k] * ur;
                                }
                                Kp[2 * (k * 6 + comp)] += vr;
                                Kp[2 * (k * 6 + comp) + 1] += vi;
                            }
                        }
                }
            }
            free(wbuf);
            free(e);
            free(work);
            free(L3);
            free(R3);
            free(L1);
            free(L2);
            free(R1);
            free(R2);
        }
        for (int t = 0; t < nt; ++t)
            for (int i = 0; i < M * 12; ++i) K[i] += Kpart[(size_t)t * M * 12 + i];
        free(Kpart);
        free(lstore);
        free(rstore);
    }
    for (int i = 0; i < M * 12; ++i) K[i] /= (double)R;

    /* Ascending energies and the result (:612-659). */
    double* eps_sorted = (double*)malloc(sizeof(double) * M);
    for (int k = 0; k < M; ++k) {
        const int src = M - 1 - k;
        const double th = M_PI * ((double)src + 0.5) / (double)M;
        eps_sorted[k] = cos(th);
        energy_out[k] = op->center + op->half_width * eps_sorted[k];
    }
    if (formulation == 0) {
        for (int k = 0; k < M; ++k) {
            const int src = M - 1 - k;
            for (int c = 0; c < 6; ++c) sigma_out[k * 6 + c] = prefactor * K[2 * (src * 6 + c)];
        }
    } else {
        double running[6] = {0, 0, 0, 0, 0, 0}, prev[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < M; ++k) {
            const int src = M - 1 - k;
            double integrand[6];
            for (int c = 0; c < 6; ++c) integrand[c] = -K[2 * (src * 6 + c) + 1]; /* Re(i z) */
            if (k > 0) {
                const double de = eps_sorted[k] - eps_sorted[k - 1];
                for (int c = 0; c < 6; ++c) running[c] += 0.5 * (prev[c] + integrand[c]) * de;
            }
            for (int c = 0; c < 6; ++c) {
                sigma_out[k * 6 + c] = prefactor * running[c];
                prev[c] = integrand[c];
            }
        }
    }
    free(eps_sorted);
    for (int a = 0; a < 3; ++a) {
        free(rinit[a]);
        free(rprev[a]);
        free(rcurr[a]);
        free(rnext[a]);
        free(laxes[a]);
    }
    free(lprev);
    free(lcurr);
    free(lnext);
    free(tmp);
    free(K);
    free(g);
    free(phi3w);
    free(pw);
    free(pwm);
    free(eps);
    free(root);
    return 0;
}

/* Raw Philox-4x32-10 block, for the published known-answer vectors. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox(c, key[0], key[1]);
    for (int i = 0; i < 4; ++i) out[i] = c[i];
}
