// psg_pipe_f64.cu — the float64 instantiations of the generic
// pipeline_kernel (largest radix 8, with and without the next-row bulk
// prefetch), and the form whose work areas are in global memory (long
// traces).
#include "psg_kernel.cuh"

namespace psg {

const void* pipe_kernel_f64(int recipe, bool pf) {
  if (recipe != RC_GENERIC) return recipe_kernel_f64(recipe, pf);
  return pf ? (const void*)pipeline_kernel<double, 8, true, false, RC_GENERIC>
            : (const void*)pipeline_kernel<double, 8, false, false, RC_GENERIC>;
}

const void* wide_kernel_f64() { return (const void*)pipeline_kernel<double, 8, false, false, RC_GENERIC, true>; }

}  // namespace psg
