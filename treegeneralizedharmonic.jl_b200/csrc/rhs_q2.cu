// Right-hand-side kernel instantiations for finite-difference order q = 2.
#include "rhs_inst.cuh"

namespace tgh {
TGH_DEFINE_RHS_LAUNCH(2, f64, double)
}  // namespace tgh
