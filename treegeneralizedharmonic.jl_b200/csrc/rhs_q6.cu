// Right-hand-side kernel instantiations for finite-difference order q = 6.
#include "rhs_inst.cuh"

namespace tgh {
TGH_DEFINE_RHS_LAUNCH(6, f64, double)
}  // namespace tgh
