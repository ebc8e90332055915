// Grain cut-off of the sintering operator: the per-cell sets of relevant
// grains (SinteringOperatorData::set_component_mask,
// operator_sintering_data.h:149-298) that the residual, Jacobian and
// preconditioner kernels restrict their grain terms to, and the statistic of
// relevant-grain counts the reference prints with it.
#include <string>

#include "sint_internal.h"
#include "sint_launch.h"

namespace sint
{
  // One thread per cell (lexicographic, n[0] fastest): bit b of mask[cell] is
  // set when the largest |eta_b| over the cell's 2^dim nodes exceeds tol --
  // the l-infinity norm of the cell's dof values of each order parameter
  // (operator_sintering_data.h:188-203).  The reference forms the union over
  // the cells of one SIMD batch; here every cell keeps its own set.
  __global__ void __launch_bounds__(256)
    grain_mask_kernel(const Grid g, int G, const double *__restrict__ u, double tol, uint16_t *__restrict__ mask)
  {
    const long long n_cells = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long cell    = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n_cells)
      return;
    const int i  = int(cell % g.n[0]);
    const int j  = int((cell / g.n[0]) % g.n[1]);
    const int k  = int(cell / ((long long)g.n[0] * g.n[1]));
    const int nl = g.dim == 3 ? 8 : 4;
    long long node[8];
    for (int l = 0; l < nl; ++l)
      node[l] = node_index(g, i + (l & 1), j + ((l >> 1) & 1), k + ((l >> 2) & 1));
    unsigned bits = 0;
    for (int b = 0; b < G; ++b)
      {
        const double *eta = u + (2 + b) * g.ld;
        double        mx  = 0.0;
        for (int l = 0; l < nl; ++l)
          mx = fmax(mx, fabs(eta[node[l]]));
        if (mx > tol)
          bits |= 1u << b;
      }
    mask[cell] = (uint16_t)bits;
  }

  // counts[k] += number of cells with k relevant grains (integer atomics:
  // the totals do not depend on the order).
  __global__ void __launch_bounds__(256)
    grain_count_kernel(long long n_cells, const uint16_t *__restrict__ mask, unsigned long long *__restrict__ counts)
  {
    __shared__ unsigned int h[SINT_MAX_GRAINS + 1];
    if (threadIdx.x <= SINT_MAX_GRAINS)
      h[threadIdx.x] = 0;
    __syncthreads();
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n_cells;
         c += (long long)gridDim.x * blockDim.x)
      atomicAdd(&h[__popc((unsigned)mask[c])], 1u);
    __syncthreads();
    if (threadIdx.x <= SINT_MAX_GRAINS && h[threadIdx.x] != 0)
      atomicAdd(&counts[threadIdx.x], (unsigned long long)h[threadIdx.x]);
  }

  static long long cell_count(const Ctx *c) { return (long long)c->grid.n[0] * c->grid.n[1] * c->grid.n[2]; }
} // namespace sint

using namespace sint;

int sint_set_component_mask(sint_ctx *c, const double *u, double tol, sint_stream_t stream)
{
  if (!c)
    {
      set_error("null context");
      return SINT_ERR_ARG;
    }
  if (!(tol >= 0.0))
    {
      set_error("sint_set_component_mask: the tolerance must be >= 0");
      return SINT_ERR_ARG;
    }
  if (tol == 0.0)
    {
      // GrainCutOffTolerance = 0 keeps every grain everywhere (driver.h:2212)
      c->cut     = false;
      c->cut_tol = 0.0;
      return SINT_OK;
    }
  if (!u || (reinterpret_cast<uintptr_t>(u) & 15u) != 0)
    {
      set_error("sint_set_component_mask: u must be a 16-byte aligned device pointer");
      return SINT_ERR_ARG;
    }
  cudaError_t e = cudaSuccess;
  if (!c->mask)
    {
      c->n_cells = cell_count(c);
      if ((e = cudaMalloc(&c->mask, sizeof(uint16_t) * (size_t)c->n_cells)) != cudaSuccess)
        {
          c->mask = nullptr;
          return cuda_fail(e, "sint_set_component_mask: allocation");
        }
    }
  const long long nb = (c->n_cells + 255) / 256;
  grain_mask_kernel<<<dim3((unsigned)nb), 256, 0, stream>>>(c->grid, c->G, u, tol, c->mask);
  count_launches(1);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return cuda_fail(e, "sint_set_component_mask");
  c->cut     = true;
  c->cut_tol = tol;
  return SINT_OK;
}

int sint_component_mask_statistics(sint_ctx *c, int64_t *counts, sint_stream_t stream)
{
  if (!c || !counts)
    {
      set_error("sint_component_mask_statistics: null argument");
      return SINT_ERR_ARG;
    }
  if (!c->cut)
    {
      set_error("sint_component_mask_statistics: no grain cut-off set");
      return SINT_ERR_NOT_READY;
    }
  // the reduction buffer is free between operator calls on this context
  unsigned long long *d = reinterpret_cast<unsigned long long *>(c->red);
  unsigned long long  h[SINT_MAX_GRAINS + 1];
  cudaError_t         e = cudaMemsetAsync(d, 0, sizeof(h), stream);
  if (e == cudaSuccess)
    {
      grain_count_kernel<<<dim3(4 * 148), 256, 0, stream>>>(c->n_cells, c->mask, d);
      count_launches(1);
      e = cudaGetLastError();
    }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_component_mask_statistics");
  for (int k = 0; k <= c->G; ++k)
    counts[k] = (int64_t)h[k];
  return SINT_OK;
}

int sint_get_component_mask(const sint_ctx *c, uint16_t *dst, sint_stream_t stream)
{
  if (!c || !dst)
    {
      set_error("sint_get_component_mask: null argument");
      return SINT_ERR_ARG;
    }
  if (!c->cut)
    {
      set_error("sint_get_component_mask: no grain cut-off set");
      return SINT_ERR_NOT_READY;
    }
  const cudaError_t e =
    cudaMemcpyAsync(dst, c->mask, sizeof(uint16_t) * (size_t)c->n_cells, cudaMemcpyDeviceToDevice, stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_get_component_mask");
  return SINT_OK;
}
