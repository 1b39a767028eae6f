// Kernel-smoothed density from KPM moments, rsatb::calc::evaluate_kpm_density
// (rsatb/calc/kpm.hpp:206-241) with the weights of kpm_kernel_weights
// (:52-85, jackson_kernel :18-26).  One thread per energy point, T_n(x) by
// the three-term recurrence in FP64.
#include "common.cuh"

#include <cmath>
#include <vector>

namespace rsatb_b200 {

// g_n, n < n_moments, for the summation kernels of kpm.hpp:52-85.
void kpm_kernel_weights(int kernel, int n, double* g) {
    for (int i = 0; i < n; ++i) g[i] = 1.0;
    if (kernel == RSATB_KPM_JACKSON) {
        const double denom = double(n + 1);
        const double theta = M_PI / denom;
        const double cot_theta = std::cos(theta) / std::sin(theta);
        g[0] = 1.0;
        for (int i = 1; i < n; ++i)
            g[i] = ((denom - i) * std::cos(theta * i) + cot_theta * std::sin(theta * i)) / denom;
    } else if (kernel == RSATB_KPM_COSTAPER) {
        const int n0 = n / 2;
        for (int i = n0; i < n; ++i) {
            const double s = double(i - n0) / double(n - n0);
            g[i] = 0.5 * (1.0 + std::cos(M_PI * s));
        }
    } else if (kernel == RSATB_KPM_VPTAPER) {
        const int n0 = n / 2;
        for (int i = n0; i < n; ++i) g[i] = double(n - i) / double(n - n0);
    }
}

namespace {

__global__ void kpm_density_kernel(const double* __restrict__ gmu, int n_moments,
                                   const double* __restrict__ x, int nx, double edge_inset,
                                   double* __restrict__ rho) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nx) return;
    const double xj = fmax(-1.0 + edge_inset, fmin(1.0 - edge_inset, x[j]));
    double t_prev = 1.0, t_curr = xj;
    double acc = gmu[0];
    if (n_moments > 1) acc += 2.0 * gmu[1] * t_curr;
    for (int n = 2; n < n_moments; ++n) {
        const double t_next = 2.0 * xj * t_curr - t_prev;
        acc += 2.0 * gmu[n] * t_next;
        t_prev = t_curr;
        t_curr = t_next;
    }
    rho[j] = acc / (M_PI * sqrt(fmax(1e-14, 1.0 - xj * xj)));
}

}  // namespace
}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" int rsatb_evaluate_kpm_density(rsatb_ctx_t ctx, const double* moments, int n_moments,
                                          const double* x, int nx, double edge_inset, int kernel,
                                          double* rho_out) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (nx < 0 || n_moments < 0 || (nx > 0 && (!x || !rho_out)) || (n_moments > 0 && !moments))
        return set_error(RSATB_INVALID_ARGUMENT, "evaluate_kpm_density: bad arguments");
    if (kernel < RSATB_KPM_NONE || kernel > RSATB_KPM_VPTAPER)
        return set_error(RSATB_INVALID_ARGUMENT, "unknown KPM kernel %d", kernel);
    if (nx == 0) return RSATB_SUCCESS;
    if (n_moments == 0) {
        for (int j = 0; j < nx; ++j) rho_out[j] = 0.0;
        return RSATB_SUCCESS;
    }
    // g_n * Re(mu_n) on the host: n_moments products, as kpm.hpp forms them.
    std::vector<double> g(n_moments), gmu(n_moments);
    kpm_kernel_weights(kernel, n_moments, g.data());
    for (int n = 0; n < n_moments; ++n) gmu[n] = g[n] * moments[2 * n];
    double *d_gmu = nullptr, *d_x = nullptr, *d_rho = nullptr;
    RSATB_CUDA_TRY(cudaMallocAsync(&d_gmu, sizeof(double) * n_moments, ctx->stream));
    RSATB_CUDA_TRY(cudaMallocAsync(&d_x, sizeof(double) * nx, ctx->stream));
    RSATB_CUDA_TRY(cudaMallocAsync(&d_rho, sizeof(double) * nx, ctx->stream));
    RSATB_CUDA_TRY(cudaMemcpyAsync(d_gmu, gmu.data(), sizeof(double) * n_moments,
                                   cudaMemcpyHostToDevice, ctx->stream));
    RSATB_CUDA_TRY(cudaMemcpyAsync(d_x, x, sizeof(double) * nx, cudaMemcpyHostToDevice,
                                   ctx->stream));
    const int threads = 128;
    kpm_density_kernel<<<(nx + threads - 1) / threads, threads, 0, ctx->stream>>>(
        d_gmu, n_moments, d_x, nx, edge_inset, d_rho);
    RSATB_LAUNCH_CHECK(ctx);
    RSATB_CUDA_TRY(cudaMemcpyAsync(rho_out, d_rho, sizeof(double) * nx, cudaMemcpyDeviceToHost,
                                   ctx->stream));
    cudaFreeAsync(d_gmu, ctx->stream);
    cudaFreeAsync(d_x, ctx->stream);
    cudaFreeAsync(d_rho, ctx->stream);
    RSATB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return RSATB_SUCCESS;
}
