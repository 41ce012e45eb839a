// psg_pipe_f32.cu — the float32 instantiations of the generic pipeline_kernel
// (any step sequence): with and without the next-row bulk prefetch,
// single-job and batched (several plans and blocks per launch), and the
// single-job form whose work areas are in global memory (long traces).
#include "psg_kernel.cuh"

namespace psg {

const void* pipe_kernel_f32(int recipe, bool pf, bool batch) {
  if (recipe != RC_GENERIC && !batch) return recipe_kernel_f32(recipe, pf);
  if (batch)
    return pf ? (const void*)pipeline_kernel<float, 12, true, true, RC_GENERIC>
              : (const void*)pipeline_kernel<float, 12, false, true, RC_GENERIC>;
  return pf ? (const void*)pipeline_kernel<float, 12, true, false, RC_GENERIC>
            : (const void*)pipeline_kernel<float, 12, false, false, RC_GENERIC>;
}

const void* wide_kernel_f32() { return (const void*)pipeline_kernel<float, 12, false, false, RC_GENERIC, true>; }

}  // namespace psg
