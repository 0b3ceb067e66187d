// Right-hand-side kernel instantiations for finite-difference order q = 6, mixed form.
#include "rhs_inst.cuh"

namespace tgh {
TGH_DEFINE_RHS_LAUNCH(6, f32, float)
}  // namespace tgh
