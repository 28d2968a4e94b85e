// Fused explicit-stencil RHS kernels (placeholder until the z-marching kernels land).
#include <stdexcept>

#include "cruna_internal.cuh"

namespace cruna {

bool fused_supported(const cruna_ctx *) { return false; }

void rhs_direct_fused(cruna_ctx *, const double *, double *, int, const double *, double *, double *,
                      double) {
  throw std::runtime_error("fused RHS path is not available");
}

}  // namespace cruna
