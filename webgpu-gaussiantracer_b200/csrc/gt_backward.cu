// gt_backward.cu — adjoint of the tracer (placeholder until the adjoint kernel lands).
#include "gt_internal.cuh"

extern "C" gt_status gt_backward(gt_context*, const gt_scene*, const gt_uniforms*, uint32_t, uint32_t, const float*,
                                 float*, uint32_t, gt_bwd_opts*, gt_render_stats*) {
  return GT_ERR_UNSUPPORTED;
}
extern "C" gt_status gt_backward_batch(gt_context*, const gt_batch_item*, uint32_t, const gt_scene* const*,
                                       float* const*, uint32_t, uint32_t, gt_bwd_opts*, gt_render_stats*) {
  return GT_ERR_UNSUPPORTED;
}
