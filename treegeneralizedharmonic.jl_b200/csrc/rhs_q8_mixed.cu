// Right-hand-side kernel instantiations for finite-difference order q = 8, mixed form.
#include "rhs_inst.cuh"

namespace tgh {
TGH_DEFINE_RHS_LAUNCH(8, f32, float)
}  // namespace tgh
