// psg_recipe_f32.cu — the float32 recipe instantiations of pipeline_kernel
// (fixed step sequences as straight-line code), with and without the
// next-row bulk prefetch.
#include "psg_kernel.cuh"

namespace psg {

template <int R> static const void* pick_f32(bool pf) {
  return pf ? (const void*)pipeline_kernel<float, 12, true, false, R>
            : (const void*)pipeline_kernel<float, 12, false, false, R>;
}

const void* recipe_kernel_f32(int recipe, bool pf) {
  switch (recipe) {
    case RC_DFA: return pick_f32<RC_DFA>(pf);
    case RC_DFAN: return pick_f32<RC_DFAN>(pf);
    case RC_FN: return pick_f32<RC_FN>(pf);
    case RC_FG: return pick_f32<RC_FG>(pf);
    default: return nullptr;
  }
}

}  // namespace psg
