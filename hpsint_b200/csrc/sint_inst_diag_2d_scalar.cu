// Instantiates the preconditioner-diagonal kernels for dim = 2, scalar mobility, G = 1..12.
#include "sint_launch_impl.cuh"

namespace sint
{
  template cudaError_t launch_diag<2, false>(int, const Grid &, const Phys &, const double *, double *, double *,
                                            const uint16_t *, const AdvData *, cudaStream_t);
} // namespace sint
