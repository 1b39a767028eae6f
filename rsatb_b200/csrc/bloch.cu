// Bloch sums of real-space operator images at one k-point.
//
// The reference assembles H(k) entry by entry: for every bond (i, j, R) it
// multiplies the block by the Bloch phase exp(-2 pi i k . R) (BlochPhase,
// rsatb/operator/block_assembly.hpp:31-38) and adds it into block (i, j)
// (AddLocalBlock, :66-100).  The velocity of the commutator form takes the
// same sum with the extra factor i (R + r_j - r_i)_a per bond
// (AccumulateBondMoment, rsatb/operator/commutator_velocity.hpp:114-225).
//
// Here the bonds are kept on the device sorted by their output block, with
// slot_ptr marking each block's run, so one warp sums one output block in a
// fixed order (deterministic, no atomics): the lanes hold the block's
// elements and every lane forms the same phase with sincospi.
#include "common.cuh"

#include <algorithm>

namespace rsatb_b200 {
namespace {

template <bool CPLX_IN>
__global__ void bloch_sum_kernel(int64_t n_slots, const int64_t* __restrict__ slot_ptr,
                                 const double* __restrict__ shifts, const double* __restrict__ vals,
                                 const double* __restrict__ weights, int bb, double kx, double ky,
                                 double kz, int imag_unit, double2* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t s = warp; s < n_slots; s += n_warps) {
        const int64_t e0 = slot_ptr[s], e1 = slot_ptr[s + 1];
        for (int l0 = 0; l0 < bb; l0 += 32) {
            const int l = l0 + lane;
            double ar = 0.0, ai = 0.0;
            for (int64_t e = e0; e < e1; ++e) {
                const double x = shifts[3 * e] * kx + shifts[3 * e + 1] * ky + shifts[3 * e + 2] * kz;
                double sn, cs;
                sincospi(-2.0 * x, &sn, &cs);  // exp(-2 pi i k . R)
                const double w = weights ? weights[e] : 1.0;
                double pr = cs * w, pi = sn * w;
                if (imag_unit) {  // times i
                    const double t = pr;
                    pr = -pi;
                    pi = t;
                }
                if (l < bb) {
                    if constexpr (CPLX_IN) {
                        const double vr = vals[2 * (e * bb + l)], vi = vals[2 * (e * bb + l) + 1];
                        ar += pr * vr - pi * vi;
                        ai += pr * vi + pi * vr;
                    } else {
                        const double v = vals[e * bb + l];
                        ar += pr * v;
                        ai += pi * v;
                    }
                }
            }
            if (l < bb) out[s * bb + l] = make_double2(ar, ai);
        }
    }
}

}  // namespace
}  // namespace rsatb_b200

using namespace rsatb_b200;

extern "C" int rsatb_bloch_sum(rsatb_ctx_t ctx, rsatb_bsr_t out, const int64_t* slot_ptr,
                               const double* shifts, const void* image_values,
                               rsatb_dtype image_dtype, const double* weights, const double* k,
                               int imag_unit) {
    clear_error();
    RSATB_TRY(check_ctx(ctx));
    if (!out || !slot_ptr || !k || (out->nnz_blocks > 0 && (!shifts || !image_values)))
        return set_error(RSATB_INVALID_ARGUMENT, "bloch_sum: null argument");
    if (out->dtype != RSATB_C128)
        return set_error(RSATB_INVALID_ARGUMENT, "bloch_sum: the output matrix must be C128");
    if (image_dtype != RSATB_F64 && image_dtype != RSATB_C128)
        return set_error(RSATB_INVALID_ARGUMENT, "bloch_sum: images must be F64 or C128");
    if (out->flags & RSATB_BSR_IMAGINARY_UNIT)
        return set_error(RSATB_INVALID_ARGUMENT, "bloch_sum: output carries the imaginary-unit flag");
    const int64_t n_slots = out->nnz_blocks;
    if (n_slots == 0) return RSATB_SUCCESS;
    const int bb = out->block_size * out->block_size;
    const int threads = 256;
    const int64_t warps_needed = n_slots;
    const int64_t grid = std::min<int64_t>((warps_needed * 32 + threads - 1) / threads,
                                           int64_t(ctx->sm_count) * 16);
    if (image_dtype == RSATB_C128)
        bloch_sum_kernel<true><<<unsigned(grid), threads, 0, ctx->stream>>>(
            n_slots, slot_ptr, shifts, static_cast<const double*>(image_values), weights, bb,
            k[0], k[1], k[2], imag_unit ? 1 : 0, static_cast<double2*>(out->values));
    else
        bloch_sum_kernel<false><<<unsigned(grid), threads, 0, ctx->stream>>>(
            n_slots, slot_ptr, shifts, static_cast<const double*>(image_values), weights, bb,
            k[0], k[1], k[2], imag_unit ? 1 : 0, static_cast<double2*>(out->values));
    RSATB_LAUNCH_CHECK(ctx);
    return RSATB_SUCCESS;
}
