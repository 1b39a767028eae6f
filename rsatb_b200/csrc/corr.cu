// Time-propagation coefficients and the correlation-series DOS.
//
// rsatb::calc::timeprop_coeff (rsatb/calc/cheby.hpp:85-106) expands
// e^{-i x t} = sum_n (2 - delta_n0) (-i)^n J_n(t) T_n(x), truncated by
// build_bessel_vector (rsatb/calc/bessel.hpp:9-52): terms n = 0, 1, ... up
// to, not including, the first n with |J_n(t)| <= eps and |J_{n+1}(t)| <= eps.
// corr_from_moments (rsatb/calc/dos.hpp:30-46) sums the moments with these
// coefficients at t_j = j pi, j = 1..nt, which gives the overlap
// C(t_j) = <psi| e^{-i Op t_j} |psi>; ComputeDos "corr"
// (rsatb/calc/observables.hpp:393-428) applies a Hann window, mirrors the
// series to negative times and takes an unnormalised inverse FFT of 2 nt
// points.
//
// The Bessel values come from Miller's backward recurrence
// J_{n-1} = (2n / t) J_n - J_{n+1}, started well above the truncation order
// with an arbitrary value and normalised by J_0 + 2 sum_k J_2k = 1 (the
// method of Miller, as in Abramowitz and Stegun 9.12 and Numerical Recipes
// 6.5).  One thread handles one time: a first pass finds the normalisation,
// a second pass repeats the identical arithmetic (so both passes rescale at
// the same orders) and applies the truncation rule and the sum.  Values are
// kept below 2^600 by exact power-of-two rescaling.
#include "common.cuh"

#include <cufft.h>

#include <cmath>
#include <vector>

namespace rsatb_b200 {
namespace {

constexpr int kRescaleExp = 600;
constexpr int kMaxOrder = 65536;  // bessel.hpp:21 gives up at this order

// First order of the backward recurrence: past the turning point n = t by
// 30 t^(1/3) + 60, where J_n(t) is below 1e-60 for every t >= pi.
__host__ __device__ inline int miller_start(double t) {
    return int(t + 30.0 * cbrt(t) + 60.0);
}

// Runs the backward recurrence for time t.  Pass 1 (coeff == nullptr and
// mu == nullptr): returns the normalisation sum in *norm and the rescale
// count in *k_total.  Pass 2: with the normalisation known, finds the
// truncation and either writes the coefficients (coeff, capacity cap) or
// sums them against the moments (mu, n_mu) into *sum.  Returns the number
// of terms, or -1 when the start order was not far enough out (never for
// the start above; the check keeps a wrong start from passing silently).
__device__ int miller_pass(double t, double eps, int forward, double* norm, int* k_total,
                           double2* coeff, int cap, const double2* mu, int n_mu, double2* sum) {
    const int n0 = miller_start(t);
    const bool second = coeff != nullptr || mu != nullptr;
    double f = 1.0, fp1 = 0.0;  // f_n, f_{n+1} (unnormalised)
    double acc_norm = 0.0;
    int k = 0;
    const double inv_norm = second ? 1.0 / *norm : 0.0;
    const int K = second ? *k_total : 0;
    double j_next = 0.0;  // normalised J_{n+1}
    int n_terms = -1;     // set at the first order (descending) where the rule fails
    double sr = 0.0, si = 0.0;
    for (int n = n0; n >= 0; --n) {
        if (!second) {
            if ((n & 1) == 0) acc_norm += (n == 0 ? 1.0 : 2.0) * f;
        } else {
            const double jn = ldexp(f, -kRescaleExp * (K - k)) * inv_norm;
            if (n_terms < 0) {
                const bool tail = fabs(jn) <= eps && fabs(j_next) <= eps;
                if (!tail) {
                    if (n == n0) return -1;
                    n_terms = n + 1;
                }
            }
            if (n_terms >= 0) {
                // (2 - delta_n0) (-i)^n J_n forward, (+i)^n backward.
                const double m = (n == 0 ? 1.0 : 2.0) * jn;
                const int q = forward ? ((4 - (n & 3)) & 3) : (n & 3);  // power of +i
                const double cr = q == 0 ? m : (q == 2 ? -m : 0.0);
                const double ci = q == 1 ? m : (q == 3 ? -m : 0.0);
                if (coeff && n < cap) coeff[n] = make_double2(cr, ci);
                if (mu && n < n_mu) {
                    const double2 u = mu[n];
                    sr += cr * u.x - ci * u.y;
                    si += cr * u.y + ci * u.x;
                }
            }
            j_next = jn;
        }
        if (n > 0) {
            // Explicit fma: both passes must produce the same f sequence.
            const double fm1 = fma(2.0 * n / t, f, -fp1);
            fp1 = f;
            f = fm1;
            if (fabs(f) > 0x1p600) {
                f = ldexp(f, -kRescaleExp);
                fp1 = ldexp(fp1, -kRescaleExp);
                if (!second) acc_norm = ldexp(acc_norm, -kRescaleExp);
                ++k;
            }
        }
    }
    if (!second) {
        *norm = acc_norm;
        *k_total = k;
        return 0;
    }
    if (sum) *sum = make_double2(sr, si);
    return n_terms < 0 ? 0 : n_terms;
}

__global__ void timeprop_coeff_kernel(double t, double eps, int forward, double2* coeff,
                                      int cap, int* n_out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double norm = 0.0;
    int K = 0;
    miller_pass(t, eps, forward, &norm, &K, nullptr, 0, nullptr, 0, nullptr);
    *n_out = miller_pass(t, eps, forward, &norm, &K, coeff, cap, nullptr, 0, nullptr);
}

// cdos[j] = sum_{n < min(terms(j pi), n_mu)} c_n(j pi) mu_n, j = 1..nt;
// cdos[0] = mu_0 (dos.hpp:33-44).  bad is set when a start order was short.
__global__ void corr_series_kernel(const double2* __restrict__ mu, int n_mu, int nt, double eps,
                                   double2* __restrict__ cdos, int* bad) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > nt) return;
    if (j == 0) {
        cdos[0] = mu[0];
        return;
    }
    const double t = j * M_PI;
    double norm = 0.0;
    int K = 0;
    miller_pass(t, eps, 1, &norm, &K, nullptr, 0, nullptr, 0, nullptr);
    double2 s = make_double2(0.0, 0.0);
    const int n = miller_pass(t, eps, 1, &norm, &K, nullptr, 0, mu, n_mu, &s);
    if (n < 0) atomicOr(bad, 1);
    cdos[j] = s;
}

// The windowed, mirrored series of observables.hpp:405-412: full[0] = C_0;
// for i = 1..nt, w_i = (1 + cos(pi (i - 1) / nt)) / 2, full[i] = C_i w_i and
// full[2nt - i] = conj(C_i) w_i (at i = nt the mirrored value is the one
// kept, as in the reference's order of assignment).
__global__ void corr_window_kernel(const double2* __restrict__ cdos, int nt,
                                   double2* __restrict__ full) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * nt) return;
    if (i == 0) {
        full[0] = cdos[0];
        return;
    }
    if (i >= nt) {
        const int s = 2 * nt - i;  // full[i] = conj(C_s) w_s
        const double w = 0.5 * (1.0 + cos(M_PI * (s - 1) / nt));
        full[i] = make_double2(cdos[s].x * w, -cdos[s].y * w);
    } else {
        const double w = 0.5 * (1.0 + cos(M_PI * (i - 1) / nt));
        full[i] = make_double2(cdos[i].x * w, cdos[i].y * w);
    }
}

// dos[i] = Re F[nt + i], dos[nt + i] = Re F[i], i < nt (observables.hpp:421-425).
__global__ void corr_reorder_kernel(const double2* __restrict__ F, int nt, double* __restrict__ dos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * nt) return;
    dos[i] = i < nt ? F[nt + i].x : F[i - nt].x;
}

}  // namespace
}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" int rsatb_timeprop_coeff(rsatb_ctx_t ctx, double time_step, double precision,
                                    int forward, int capacity, double* coeffs, int* n_coeffs) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!n_coeffs || capacity < 0 || (capacity > 0 && !coeffs) || !(precision > 0.0) ||
        !(time_step > 0.0) || !std::isfinite(time_step))
        return set_error(RSATB_INVALID_ARGUMENT, "timeprop_coeff: bad arguments");
    if (miller_start(time_step) >= kMaxOrder)
        return set_error(RSATB_INVALID_ARGUMENT, "bessel: series not converged (time %g)",
                         time_step);
    const int cap = capacity;
    double2* d_c = nullptr;
    int* d_n = nullptr;
    RSATB_CUDA_TRY(cudaMallocAsync(&d_c, sizeof(double2) * (cap > 0 ? cap : 1), ctx->stream));
    RSATB_CUDA_TRY(cudaMallocAsync(&d_n, sizeof(int), ctx->stream));
    timeprop_coeff_kernel<<<1, 1, 0, ctx->stream>>>(time_step, precision, forward ? 1 : 0, d_c,
                                                    cap, d_n);
    RSATB_LAUNCH_CHECK(ctx);
    int n = 0;
    RSATB_CUDA_TRY(cudaMemcpyAsync(&n, d_n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (n > 0 && cap > 0)
        RSATB_CUDA_TRY(cudaMemcpyAsync(coeffs, d_c, sizeof(double2) * (n < cap ? n : cap),
                                       cudaMemcpyDeviceToHost, ctx->stream));
    cudaFreeAsync(d_c, ctx->stream);
    cudaFreeAsync(d_n, ctx->stream);
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (n < 0) return set_error(RSATB_NUMERICAL_FAILURE, "timeprop_coeff: short Miller start");
    *n_coeffs = n;
    return RSATB_SUCCESS;
}

extern "C" int rsatb_corr_dos(rsatb_ctx_t ctx, const double* moments, int n_moments, int nt,
                              double precision, double* cdos_out, double* dos_out) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!moments || n_moments < 1 || nt < 1 || !(precision > 0.0))
        return set_error(RSATB_INVALID_ARGUMENT, "corr_dos: bad arguments");
    if (miller_start(nt * M_PI) >= kMaxOrder)
        return set_error(RSATB_INVALID_ARGUMENT, "bessel: series not converged (nt %d)", nt);
    const size_t n_full = size_t(2) * nt;
    double2 *d_mu = nullptr, *d_c = nullptr, *d_full = nullptr;
    double* d_dos = nullptr;
    int* d_bad = nullptr;
    RSATB_CUDA_TRY(cudaMallocAsync(&d_mu, sizeof(double2) * n_moments, ctx->stream));
    RSATB_CUDA_TRY(cudaMallocAsync(&d_c, sizeof(double2) * (nt + 1), ctx->stream));
    RSATB_CUDA_TRY(cudaMallocAsync(&d_full, sizeof(double2) * n_full, ctx->stream));
    RSATB_CUDA_TRY(cudaMallocAsync(&d_dos, sizeof(double) * n_full, ctx->stream));
    RSATB_CUDA_TRY(cudaMallocAsync(&d_bad, sizeof(int), ctx->stream));
    RSATB_CUDA_TRY(cudaMemsetAsync(d_bad, 0, sizeof(int), ctx->stream));
    RSATB_CUDA_TRY(cudaMemcpyAsync(d_mu, moments, sizeof(double2) * n_moments,
                                   cudaMemcpyHostToDevice, ctx->stream));
    const int threads = 64;
    corr_series_kernel<<<(nt + 1 + threads - 1) / threads, threads, 0, ctx->stream>>>(
        d_mu, n_moments, nt, precision, d_c, d_bad);
    RSATB_LAUNCH_CHECK(ctx);
    corr_window_kernel<<<unsigned((n_full + 255) / 256), 256, 0, ctx->stream>>>(d_c, nt, d_full);
    RSATB_LAUNCH_CHECK(ctx);
    cufftHandle plan;
    if (cufftPlan1d(&plan, int(n_full), CUFFT_Z2Z, 1) != CUFFT_SUCCESS)
        return set_error(RSATB_CUDA_ERROR, "corr_dos: cuFFT plan of %d points failed",
                         int(n_full));
    cufftSetStream(plan, ctx->stream);
    const cufftResult fr = cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(d_full),
                                        reinterpret_cast<cufftDoubleComplex*>(d_full),
                                        CUFFT_INVERSE);
    if (fr != CUFFT_SUCCESS) {
        cufftDestroy(plan);
        return set_error(RSATB_CUDA_ERROR, "corr_dos: cuFFT inverse failed (%d)", int(fr));
    }
    corr_reorder_kernel<<<unsigned((n_full + 255) / 256), 256, 0, ctx->stream>>>(d_full, nt,
                                                                                d_dos);
    RSATB_LAUNCH_CHECK(ctx);
    int bad = 0;
    RSATB_CUDA_TRY(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    if (cdos_out)
        RSATB_CUDA_TRY(cudaMemcpyAsync(cdos_out, d_c, sizeof(double2) * (nt + 1),
                                       cudaMemcpyDeviceToHost, ctx->stream));
    if (dos_out)
        RSATB_CUDA_TRY(cudaMemcpyAsync(dos_out, d_dos, sizeof(double) * n_full,
                                       cudaMemcpyDeviceToHost, ctx->stream));
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    cufftDestroy(plan);
    cudaFreeAsync(d_mu, ctx->stream);
    cudaFreeAsync(d_c, ctx->stream);
    cudaFreeAsync(d_full, ctx->stream);
    cudaFreeAsync(d_dos, ctx->stream);
    cudaFreeAsync(d_bad, ctx->stream);
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (bad) return set_error(RSATB_NUMERICAL_FAILURE, "corr_dos: short Miller start");
    return RSATB_SUCCESS;
}

// ---------------------------------------------------------------------------
// sigma(mu, T) from a zero-temperature spectrum, integrate_dc_spectrum
// (rsatb/calc/fftcheb_transport.hpp:950-1040): at T <= 0 linear
// interpolation at mu (clamped to the ends); at T > 0 the piecewise-linear
// spectrum integrated exactly against -df/dE, interval by interval, with
// the antiderivative E - kT softplus((E - mu)/kT) of f.  One thread per
// tensor component sums its intervals in energy order.

namespace rsatb_b200 {
namespace {

constexpr double kBoltzmannEv = 8.617333262e-5;  // eV / K

__device__ double fermi_dirac_dev(double e, double mu, double temp) {
    if (temp <= 0.0) return e <= mu ? 1.0 : 0.0;
    const double beta = 1.0 / (temp * kBoltzmannEv);
    if (e >= mu) {
        const double t = exp(beta * (mu - e));
        return t / (1.0 + t);
    }
    const double t = exp(beta * (e - mu));
    return 1.0 / (1.0 + t);
}

__global__ void integrate_dc_kernel(const double* __restrict__ sigma,
                                    const double* __restrict__ energy, int n, double mu,
                                    double temp, double* __restrict__ out) {
    const int comp = threadIdx.x;
    if (comp >= 6) return;
    if (temp <= 0.0) {
        double v;
        if (mu <= energy[0]) {
            v = sigma[comp];
        } else if (mu >= energy[n - 1]) {
            v = sigma[(n - 1) * 6 + comp];
        } else {
            int hi = 1;  // first energy >= mu
            while (energy[hi] < mu) ++hi;
            const int lo = hi - 1;
            const double t = (mu - energy[lo]) / (energy[hi] - energy[lo]);
            v = (1.0 - t) * sigma[lo * 6 + comp] + t * sigma[hi * 6 + comp];
        }
        out[comp] = v;
        return;
    }
    const double kt = kBoltzmannEv * temp;
    auto F = [&](double e) {
        const double x = (e - mu) / kt;
        return e - kt * (fmax(x, 0.0) + log1p(exp(-fabs(x))));
    };
    double acc = 0.0;
    for (int i = 1; i < n; ++i) {
        const double e0 = energy[i - 1], e1 = energy[i], de = e1 - e0;
        const double f0 = fermi_dirac_dev(e0, mu, temp), f1 = fermi_dirac_dev(e1, mu, temp);
        const double weight = f0 - f1;
        const double moment = F(e1) - F(e0) - f1 * de;
        const double s0 = sigma[(i - 1) * 6 + comp], s1 = sigma[i * 6 + comp];
        acc += s0 * weight + (s1 - s0) / de * moment;
    }
    out[comp] = acc;
}

}  // namespace
}  // namespace rsatb_b200

extern "C" int rsatb_integrate_dc_spectrum(rsatb_ctx_t ctx, const double* sigma,
                                           const double* energy, int n_energy, double mu,
                                           double temp, double* sigma_out) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!sigma_out || n_energy < 0 || (n_energy > 0 && (!sigma || !energy)))
        return set_error(RSATB_INVALID_ARGUMENT, "integrate_dc_spectrum: bad arguments");
    for (int c = 0; c < 6; ++c) sigma_out[c] = 0.0;
    if (n_energy == 0) return RSATB_SUCCESS;
    if (temp > 0.0)
        for (int i = 1; i < n_energy; ++i)
            if (!(energy[i] - energy[i - 1] > 0.0))
                return set_error(RSATB_INVALID_ARGUMENT,
                                 "integrate_dc_spectrum: energies must be strictly ascending");
    double *d_s = nullptr, *d_e = nullptr, *d_o = nullptr;
    RSATB_CUDA_TRY(cudaMallocAsync(&d_s, sizeof(double) * 6 * n_energy, ctx->stream));
    RSATB_CUDA_TRY(cudaMallocAsync(&d_e, sizeof(double) * n_energy, ctx->stream));
    RSATB_CUDA_TRY(cudaMallocAsync(&d_o, sizeof(double) * 6, ctx->stream));
    RSATB_CUDA_TRY(cudaMemcpyAsync(d_s, sigma, sizeof(double) * 6 * n_energy,
                                   cudaMemcpyHostToDevice, ctx->stream));
    RSATB_CUDA_TRY(cudaMemcpyAsync(d_e, energy, sizeof(double) * n_energy,
                                   cudaMemcpyHostToDevice, ctx->stream));
    integrate_dc_kernel<<<1, 32, 0, ctx->stream>>>(d_s, d_e, n_energy, mu, temp, d_o);
    RSATB_LAUNCH_CHECK(ctx);
    RSATB_CUDA_TRY(cudaMemcpyAsync(sigma_out, d_o, sizeof(double) * 6, cudaMemcpyDeviceToHost,
                                   ctx->stream));
    cudaFreeAsync(d_s, ctx->stream);
    cudaFreeAsync(d_e, ctx->stream);
    cudaFreeAsync(d_o, ctx->stream);
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return RSATB_SUCCESS;
}
