// Instantiates the Jacobian-vector product kernels for dim = 3, tensorial mobility, G = 1..12, FP64 and FP32.
#include "sint_launch_impl.cuh"

namespace sint
{
  template cudaError_t launch_jvp<3, true, double>(int, const Grid &, const Phys &, const double *, const double *,
                                                   double *, double *, const CutTiles *, const AdvData *,
                                                   cudaStream_t);
  template cudaError_t launch_jvp<3, true, float>(int, const Grid &, const Phys &, const float *, const float *,
                                                  float *, float *, const CutTiles *, const AdvData *,
                                                  cudaStream_t);
} // namespace sint
