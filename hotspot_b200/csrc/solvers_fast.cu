// solvers_fast.cu -- placeholder entry points of the fast solver forms; each
// returns an error until its kernels are in place.
#include "dev_model.cuh"

namespace hsb {

int bicgstab_steady(hsb_dev_model *, const hsb_solver_opts *, hsb_stats *) {
  return set_error(HSB_E_ARG, "the BiCGStab steady solver is not available in this build");
}

}  // namespace hsb
