// Instantiates the preconditioner-diagonal kernels with the advection terms for dim = 3, tensorial mobility,
// G = 1..12, with and without the grain cut-off.
#include "sint_launch_impl.cuh"

namespace sint
{
  template <int DIM, bool TENS>
  cudaError_t launch_diag_adv(int G, const Grid &g, const Phys &p, const double *lin, double *dst, double *partial,
                              const uint16_t *mask, const AdvData &adv, cudaStream_t s)
  {
    return launch_diag_impl<DIM, TENS, true>(G, g, p, lin, dst, partial, mask, adv, s);
  }

  template cudaError_t launch_diag_adv<3, true>(int, const Grid &, const Phys &, const double *, double *, double *,
                                                 const uint16_t *, const AdvData &, cudaStream_t);
} // namespace sint
