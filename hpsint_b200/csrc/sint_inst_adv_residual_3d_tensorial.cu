// Instantiates the nonlinear-residual kernels with the advection terms for dim = 3, tensorial mobility,
// G = 1..12 (full operator) and the grain cut-off's classes 0..12, with_time_derivative 0..2.
#include "sint_launch_impl.cuh"

namespace sint
{
  template <int DIM, bool TENS>
  cudaError_t launch_residual_adv(int G, int wtd, const Grid &g, const Phys &p, const double *src,
                                  const double *const *hist, double *dst, double *partial, const CutTiles *cut,
                                  const AdvData &adv, cudaStream_t s)
  {
    return launch_residual_impl<DIM, TENS, true>(G, wtd, g, p, src, hist, dst, partial, cut, adv, s);
  }

  template cudaError_t launch_residual_adv<3, true>(int, int, const Grid &, const Phys &, const double *,
                                                     const double *const *, double *, double *, const CutTiles *,
                                                     const AdvData &, cudaStream_t);
} // namespace sint
