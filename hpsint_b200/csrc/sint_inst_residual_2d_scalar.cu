// Instantiates the nonlinear-residual kernels for dim = 2, scalar mobility, G = 1..12, with_time_derivative 0..2.
#include "sint_launch_impl.cuh"

namespace sint
{
  template cudaError_t launch_residual<2, false>(int, int, const Grid &, const Phys &, const double *,
                                                const double *const *, double *, double *, const CutTiles *,
                                                const AdvData *, cudaStream_t);
} // namespace sint
