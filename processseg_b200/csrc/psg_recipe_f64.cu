// psg_recipe_f64.cu — the float64 recipe instantiations of pipeline_kernel.
#include "psg_kernel.cuh"

namespace psg {

template <int R> static const void* pick_f64(bool pf) {
  return pf ? (const void*)pipeline_kernel<double, 8, true, false, R>
            : (const void*)pipeline_kernel<double, 8, false, false, R>;
}

const void* recipe_kernel_f64(int recipe, bool pf) {
  switch (recipe) {
    case RC_DFA: return pick_f64<RC_DFA>(pf);
    case RC_DFAN: return pick_f64<RC_DFAN>(pf);
    case RC_FN: return pick_f64<RC_FN>(pf);
    case RC_FG: return pick_f64<RC_FG>(pf);
    default: return nullptr;
  }
}

}  // namespace psg
