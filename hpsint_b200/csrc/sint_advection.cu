// Advection (rigid-body motion of the grains): the per-cell segment table and
// the per-segment velocities the residual and J v kernels read
// (AdvectionMechanism, sintering/advection.h:297-520; the terms themselves are
// in the cell kernels).
#include <cstdint>
#include <string>

#include "sint_internal.h"
#include "sint_launch.h"

namespace sint
{
  // Counts the ids outside [-1, n_segments).
  __global__ void advection_check_kernel(const int *__restrict__ ids, long long n, int n_segments,
                                         unsigned *__restrict__ bad)
  {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool      b = i < n && (ids[i] < -1 || ids[i] >= n_segments);
    const unsigned  w = __ballot_sync(0xffffffffu, b);
    if ((threadIdx.x & 31) == 0 && w)
      atomicAdd(bad, unsigned(__popc(w)));
  }
} // namespace sint

using namespace sint;

int sint_set_advection(sint_ctx *c, const int32_t *cell_segments, const double *segments, int n_segments,
                       sint_stream_t stream)
{
  if (!c)
    {
      set_error("null context");
      return SINT_ERR_ARG;
    }
  if (!cell_segments)
    {
      c->adv = false;
      return SINT_OK;
    }
  if (n_segments < 0 || (n_segments > 0 && !segments))
    {
      set_error("sint_set_advection: n_segments must be >= 0 and segments a device pointer");
      return SINT_ERR_ARG;
    }
  c->adv                  = false; // until the new table is in place
  const long long n_cells = (long long)c->grid.n[0] * c->grid.n[1] * c->grid.n[2], n_ids = n_cells * c->G;
  cudaError_t     e       = cudaSuccess;
  if (!c->adv_cells && (e = cudaMalloc(&c->adv_cells, sizeof(int) * (size_t)n_ids)) != cudaSuccess)
    {
      c->adv_cells = nullptr;
      return cuda_fail(e, "sint_set_advection: allocation");
    }
  if (n_segments > c->adv_seg_cap)
    {
      cudaFree(c->adv_segments);
      c->adv_seg_cap = 0;
      if ((e = cudaMalloc(&c->adv_segments, sizeof(double) * 9 * (size_t)n_segments)) != cudaSuccess)
        {
          c->adv_segments = nullptr;
          return cuda_fail(e, "sint_set_advection: allocation");
        }
      c->adv_seg_cap = n_segments;
    }
  if (!c->adv_error && (e = cudaMalloc(&c->adv_error, sizeof(unsigned))) != cudaSuccess)
    {
      c->adv_error = nullptr;
      return cuda_fail(e, "sint_set_advection: allocation");
    }
  unsigned bad = 0;
  if ((e = cudaMemcpyAsync(c->adv_cells, cell_segments, sizeof(int) * (size_t)n_ids, cudaMemcpyDeviceToDevice,
                           stream)) != cudaSuccess ||
      (n_segments > 0 && (e = cudaMemcpyAsync(c->adv_segments, segments, sizeof(double) * 9 * (size_t)n_segments,
                                              cudaMemcpyDeviceToDevice, stream)) != cudaSuccess) ||
      (e = cudaMemsetAsync(c->adv_error, 0, sizeof(unsigned), stream)) != cudaSuccess)
    return cuda_fail(e, "sint_set_advection: copy");
  advection_check_kernel<<<dim3((unsigned)((n_ids + 255) / 256)), 256, 0, stream>>>(c->adv_cells, n_ids, n_segments,
                                                                                    c->adv_error);
  count_launches(1);
  if ((e = cudaGetLastError()) != cudaSuccess ||
      (e = cudaMemcpyAsync(&bad, c->adv_error, sizeof(unsigned), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(stream)) != cudaSuccess)
    return cuda_fail(e, "sint_set_advection");
  if (bad)
    {
      set_error("sint_set_advection: " + std::to_string(bad) + " segment ids outside [-1, n_segments)");
      return SINT_ERR_ARG;
    }
  c->adv_view.cell_segments = c->adv_cells;
  c->adv_view.segments      = c->adv_segments;
  c->adv_view.n_segments    = n_segments;
  for (int d = 0; d < 3; ++d)
    c->adv_view.origin[d] = c->mesh.origin[d];
  c->adv = true;
  return SINT_OK;
}
