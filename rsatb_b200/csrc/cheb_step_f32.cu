// FP32 instantiations (mixed precision: FP32 matrix, panel and SpMM accumulation; FP64 rescale and dots) of the fused Chebyshev step and the column dots.
#include "cheb_step_impl.cuh"

namespace rsatb_b200 {

int launch_cheb_step_f32(rsatb_context* ctx, const rsatb_bsr_matrix* A, int vec_dtype,
                         StepArgs args) {
    return step_detail::launch_step_precision<float>(ctx, A, vec_dtype, args);
}

int launch_coldot_f32(rsatb_context* ctx, int vec_dtype, int64_t n_rows, StepArgs args) {
    return step_detail::launch_coldot_precision<float>(ctx, vec_dtype, n_rows, args);
}

}  // namespace rsatb_b200
