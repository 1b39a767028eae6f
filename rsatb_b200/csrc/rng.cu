// Seeded sample vectors: the device half of SampleVectors::initialize
// (rsatb/calc/observables.hpp:84-96), which calls vbcsr's
// set_random(seed, normalize, atom_index).
//
// vbcsr's generator is not part of the reference sources, so this library
// defines its own: every element is a pure function of
//   (seed, stable atom id, orbital within the atom, column)
// through the counter-based Philox-4x32-10 generator (Salmon, Moraes, Dror,
// Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).  Counter =
// (id low word, id high word, orbital, column), key = (seed low, seed high).
// The value therefore does not depend on the launch shape, the rank layout
// or the row order, and the CPU oracle reproduces it bit for bit: the
// random phase uses a Taylor-series sine/cosine written with explicit fma()
// on both sides instead of a math library.
#include "common.cuh"

#include <cmath>
#include <vector>

namespace rsatb_b200 {
namespace {

struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = M0 * c.x, hi0 = __umulhi(M0, c.x);
        const uint32_t lo1 = M1 * c.z, hi1 = __umulhi(M1, c.z);
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// Taylor coefficients (-1)^k/(2k+1)! and (-1)^k/(2k)!, correctly rounded.
__constant__ double kSin[12] = {-0.16666666666666666,    0.008333333333333333,
                                -0.0001984126984126984,  2.7557319223985893e-06,
                                -2.505210838544172e-08,  1.6059043836821613e-10,
                                -7.647163731819816e-13,  2.8114572543455206e-15,
                                -8.22063524662433e-18,   1.9572941063391263e-20,
                                -3.868170170630684e-23,  6.446950284384474e-26};
__constant__ double kCos[13] = {-0.5,
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

// (cos, sin) of 2*pi*u53/2^53 for a 53-bit integer u53.  Quadrant from the
// top two bits; the remaining fraction t in [0,1) of a quarter turn is
// folded to t <= 1/2 so the series argument stays within pi/4.
__device__ __forceinline__ void phase_of(uint64_t u53, double* c_out, double* s_out) {
    const unsigned quad = unsigned(u53 >> 51);
    const uint64_t f = u53 & ((uint64_t(1) << 51) - 1);
    double t = double(f) * 4.440892098500626e-16;  // 2^-51, exact
    const bool fold = t > 0.5;
    if (fold) t = 1.0 - t;                             // exact
    const double psi = __dmul_rn(t, 1.5707963267948966);
    const double z = __dmul_rn(psi, psi);
    double ps = kSin[11];
#pragma unroll
    for (int k = 10; k >= 0; --k) ps = fma(ps, z, kSin[k]);
    const double s = fma(__dmul_rn(psi, z), ps, psi);
    double pc = kCos[12];
#pragma unroll
    for (int k = 11; k >= 0; --k) pc = fma(pc, z, kCos[k]);
    const double c = fma(z, pc, 1.0);
    double cq = fold ? s : c;  // cos and sin of the in-quadrant angle
    double sq = fold ? c : s;
    switch (quad) {
        case 0: *c_out = cq; *s_out = sq; break;
        case 1: *c_out = -sq; *s_out = cq; break;
        case 2: *c_out = -cq; *s_out = -sq; break;
        default: *c_out = sq; *s_out = -cq; break;
    }
}

template <typename T>
__global__ void set_random_kernel(uint64_t seed, int kind, double scale,
                                  const int64_t* __restrict__ atom_index, int orbitals,
                                  int64_t n_rows, int n_vectors, int64_t first_column,
                                  bool complex_out, T* out) {
    const int64_t total = n_rows * n_vectors;
    const uint32_t k0 = uint32_t(seed), k1 = uint32_t(seed >> 32);
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
         e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t row = e / n_vectors;
        const int col = int(e - row * n_vectors);
        const int64_t atom = row / orbitals;
        const int orb = int(row - atom * orbitals);
        const uint64_t id = uint64_t(atom_index[atom]);
        const uint32_t gcol = uint32_t(first_column + col);
        const U4 r = philox4x32_10(U4{uint32_t(id), uint32_t(id >> 32), uint32_t(orb), gcol}, k0, k1);
        double re = 0.0, im = 0.0;
        if (kind == RSATB_RANDOM_PHASE) {
            const uint64_t u53 = (uint64_t(r.x) << 21) ^ uint64_t(r.y >> 11);
            phase_of(u53, &re, &im);
            re = __dmul_rn(re, scale);
            im = __dmul_rn(im, scale);
        } else if (kind == RSATB_RANDOM_RADEMACHER) {
            re = (r.z & 1u) ? -scale : scale;
        } else {
            const uint64_t a = (uint64_t(r.x) << 21) ^ uint64_t(r.y >> 11);
            const uint64_t b = (uint64_t(r.z) << 21) ^ uint64_t(r.w >> 11);
            re = __dmul_rn(double(int64_t(2 * a) - (int64_t(1) << 53)) * 1.1102230246251565e-16,
                           scale);
            im = __dmul_rn(double(int64_t(2 * b) - (int64_t(1) << 53)) * 1.1102230246251565e-16,
                           scale);
        }
        if (complex_out) {
            out[2 * e] = T(re);
            out[2 * e + 1] = T(im);
        } else {
            out[e] = T(re);
        }
    }
}

}  // namespace
}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" int rsatb_set_random(rsatb_ctx_t ctx, uint64_t seed, int kind, int normalize,
                                const int64_t* atom_index, int n_atoms, int orbitals_per_atom,
                                int64_t n_rows_global, int n_vectors, int64_t first_column,
                                rsatb_dtype dtype, void* out) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!atom_index || !out || n_atoms < 0 || orbitals_per_atom <= 0 || n_vectors <= 0 ||
        first_column < 0 || first_column + n_vectors > (int64_t(1) << 32) || !dtype_valid(dtype))
        return set_error(RSATB_INVALID_ARGUMENT, "set_random: bad arguments");
    if (kind < RSATB_RANDOM_PHASE || kind > RSATB_RANDOM_UNIFORM)
        return set_error(RSATB_INVALID_ARGUMENT, "set_random: unknown distribution %d", kind);
    if (kind == RSATB_RANDOM_PHASE && !dtype_is_complex(dtype))
        return set_error(RSATB_INVALID_ARGUMENT, "a random phase needs a complex multivector");
    if (normalize && n_rows_global <= 0)
        return set_error(RSATB_INVALID_ARGUMENT, "normalising needs n_rows_global > 0");
    const int64_t n_rows = int64_t(n_atoms) * orbitals_per_atom;
    if (n_rows == 0) return RSATB_SUCCESS;
    // Scale 1/sqrt(N): both operations correctly rounded, so the host value
    // is the one the oracle uses.
    const double scale = normalize ? 1.0 / std::sqrt(double(n_rows_global)) : 1.0;
    int64_t* d_ids = nullptr;
    RSATB_CUDA_TRY(cudaMallocAsync(&d_ids, sizeof(int64_t) * n_atoms, ctx->stream));
    cudaError_t err = cudaMemcpyAsync(d_ids, atom_index, sizeof(int64_t) * n_atoms,
                                      cudaMemcpyHostToDevice, ctx->stream);
    if (err != cudaSuccess) {
        cudaFreeAsync(d_ids, ctx->stream);
        return set_error(RSATB_CUDA_ERROR, "set_random upload: %s", cudaGetErrorString(err));
    }
    const int threads = 256;
    int64_t grid = (n_rows * n_vectors + threads - 1) / threads;
    if (grid > int64_t(ctx->sm_count) * 32) grid = int64_t(ctx->sm_count) * 32;
    const bool cplx = dtype_is_complex(dtype);
    if (dtype_is_double(dtype))
        set_random_kernel<double><<<unsigned(grid), threads, 0, ctx->stream>>>(
            seed, kind, scale, d_ids, orbitals_per_atom, n_rows, n_vectors, first_column, cplx,
            static_cast<double*>(out));
    else
        set_random_kernel<float><<<unsigned(grid), threads, 0, ctx->stream>>>(
            seed, kind, scale, d_ids, orbitals_per_atom, n_rows, n_vectors, first_column, cplx,
            static_cast<float*>(out));
    err = cudaGetLastError();
    cudaFreeAsync(d_ids, ctx->stream);
    if (err != cudaSuccess)
        return set_error(RSATB_CUDA_ERROR, "set_random launch: %s", cudaGetErrorString(err));
    ctx->launches++;
    return RSATB_SUCCESS;
}
