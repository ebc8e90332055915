// Instantiates the Jacobian-vector product kernels with the advection terms for dim = 2, scalar mobility,
// G = 1..12 (full operator) and the grain cut-off's classes 0..12, FP64 and FP32.
#include "sint_launch_impl.cuh"

namespace sint
{
  template <int DIM, bool TENS, typename R>
  cudaError_t launch_jvp_adv(int G, const Grid &g, const Phys &p, const R *lin, const R *src, R *dst, R *partial,
                             const CutTiles *cut, const AdvData &adv, cudaStream_t s)
  {
    return launch_jvp_impl<DIM, TENS, R, true>(G, g, p, lin, src, dst, partial, cut, adv, s);
  }

  template cudaError_t launch_jvp_adv<2, false, double>(int, const Grid &, const Phys &, const double *,
                                                        const double *, double *, double *, const CutTiles *,
                                                        const AdvData &, cudaStream_t);
  template cudaError_t launch_jvp_adv<2, false, float>(int, const Grid &, const Phys &, const float *, const float *,
                                                       float *, float *, const CutTiles *, const AdvData &,
                                                       cudaStream_t);
} // namespace sint
