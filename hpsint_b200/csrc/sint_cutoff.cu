// Grain cut-off of the sintering operator: the per-cell sets of relevant
// grains (SinteringOperatorData::set_component_mask,
// operator_sintering_data.h:149-298) that the residual, Jacobian and
// preconditioner kernels restrict their grain terms to, and the statistic of
// relevant-grain counts the reference prints with it.
//
// The reference dispatches every cell batch to the kernel instantiated for
// its number of relevant grains (EXPAND_OPERATIONS_N_COMP_NT,
// operator_sintering_generic.h:482-530).  Here the unit is a tile: tiles are
// sorted into classes by the number of grains relevant on any of their
// cells, and each class runs the kernels instantiated for that many grains
// on the compacted components.  The class offsets stay on the device, so
// the launch sequence of an operator call does not depend on the masks and
// captured CUDA graphs stay valid when they change.
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
      {
        int n[3] = {i + (l & 1), j + ((l >> 1) & 1), k + ((l >> 2) & 1)};
        for (int d = 0; d < 3; ++d)
          if (((g.periodic >> d) & 1) && n[d] == g.n[d])
            n[d] = 0; // a slave reads its periodic master, as the operator does
        node[l] = node_index(g, n[0], n[1], n[2]);
      }
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

  // One thread per tile: the union of the masks of its cells inside the
  // mesh, and the tile counted in the class of its number of grains.
  __global__ void __launch_bounds__(256)
    tile_union_kernel(const Grid g, const uint16_t *__restrict__ cell_mask, uint16_t *__restrict__ tile_union,
                      unsigned *__restrict__ count)
  {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.n_tiles)
      return;
    const int TX = g.dim == 3 ? Tile<3>::TX : Tile<2>::TX, TY = g.dim == 3 ? Tile<3>::TY : Tile<2>::TY,
              TZ = g.dim == 3 ? Tile<3>::TZ : 1;
    const int o0 = int(t % g.nt[0]) * TX, o1 = int((t / g.nt[0]) % g.nt[1]) * TY,
              o2 = int(t / ((long long)g.nt[0] * g.nt[1])) * TZ;
    unsigned u = 0;
    for (int k = o2; k < o2 + TZ && k < g.n[2]; ++k)
      for (int j = o1; j < o1 + TY && j < g.n[1]; ++j)
        for (int i = o0; i < o0 + TX && i < g.n[0]; ++i)
          u |= cell_mask[i + (long long)g.n[0] * (j + (long long)g.n[1] * k)];
    tile_union[t] = (uint16_t)u;
    atomicAdd(&count[__popc(u)], 1u);
  }

  // One thread: class offsets from the class sizes; the sizes become the
  // scatter cursors.
  __global__ void class_scan_kernel(int G, unsigned *__restrict__ count, int *__restrict__ range)
  {
    if (threadIdx.x != 0 || blockIdx.x != 0)
      return;
    int acc = 0;
    for (int k = 0; k <= SINT_MAX_GRAINS + 1; ++k)
      {
        range[k] = acc;
        if (k <= G)
          {
            const unsigned n = count[k];
            count[k]         = (unsigned)acc;
            acc += (int)n;
          }
      }
  }

  // One thread per tile: its slot in its class (the order inside a class
  // does not change any result: tiles write disjoint outputs).
  __global__ void __launch_bounds__(256)
    class_scatter_kernel(long long n_tiles, const uint16_t *__restrict__ tile_union, unsigned *__restrict__ cursor,
                         int *__restrict__ tiles, unsigned long long *__restrict__ grains,
                         uint16_t *__restrict__ sorted_union)
  {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tiles)
      return;
    const unsigned     u   = tile_union[t];
    const unsigned     pos = atomicAdd(&cursor[__popc(u)], 1u);
    unsigned long long gl  = 0;
    int                n   = 0;
    for (int b = 0; b < SINT_MAX_GRAINS; ++b)
      if ((u >> b) & 1u)
        gl |= (unsigned long long)b << (4 * n++);
    tiles[pos]        = (int)t;
    grains[pos]       = gl;
    sorted_union[pos] = (uint16_t)u;
  }

  // One thread per node: the grains relevant on any cell the node belongs to.
  // A grain outside this set gets no residual, Jacobian or preconditioner
  // entry at the node, so every GMRES vector is zero there.
  __global__ void __launch_bounds__(256)
    node_mask_kernel(const Grid g, const uint16_t *__restrict__ cell_mask, uint16_t *__restrict__ node_mask)
  {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.N)
      return;
    const int co[3] = {int(n % g.nn[0]), int((n / g.nn[0]) % g.nn[1]), int(n / ((long long)g.nn[0] * g.nn[1]))};
    // the cells around the node; across a periodic boundary a master node
    // and its slaves share the cells of both sides (the slave rows are added
    // to the master rows), so both get the same set
    int cells[3][2];
    for (int d = 0; d < 3; ++d)
      for (int o = 0; o < 2; ++o)
        {
          int c = co[d] - 1 + o;
          if ((g.periodic >> d) & 1)
            c = c < 0 ? g.n[d] - 1 : (c >= g.n[d] ? 0 : c);
          cells[d][o] = (c >= 0 && c < g.n[d]) ? c : -1;
        }
    unsigned u = 0;
    for (int ok = 0; ok < 2; ++ok)
      for (int oj = 0; oj < 2; ++oj)
        for (int oi = 0; oi < 2; ++oi)
          {
            const int ci = cells[0][oi], cj = cells[1][oj], ck = cells[2][ok];
            if (ci >= 0 && cj >= 0 && ck >= 0)
              u |= cell_mask[ci + (long long)g.n[0] * (cj + (long long)g.n[1] * ck)];
          }
    node_mask[n] = (uint16_t)u;
  }

  // One block of 32 warps per 32-bit word of the live bitmap, one warp per
  // chunk of LIVE_CHUNK elements of a block vector (C blocks of stride ld):
  // the chunk is live when one of its elements is c or mu, or a grain
  // relevant at its node.
  __global__ void __launch_bounds__(1024)
    live_chunk_kernel(const Grid g, int C, const uint16_t *__restrict__ node_mask, uint32_t *__restrict__ live,
                      long long n_words)
  {
    __shared__ uint32_t s_bits;
    const long long     word = blockIdx.x;
    const int           k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0)
      s_bits = 0u;
    __syncthreads();
    const long long n_elem = (long long)C * g.ld;
    const long long e0     = (word * 32 + k) * LIVE_CHUNK;
    if (word < n_words && e0 < n_elem) // the same for the whole warp
      {
        const long long e1 = (e0 + LIVE_CHUNK < n_elem ? e0 + LIVE_CHUNK : n_elem) - 1;
        // one division per chunk for its first block (component); a chunk
        // that starts in the c or mu block is live
        const long long b0  = e0 / g.ld;
        bool            any = b0 < 2;
        if (!any)
          for (long long e = e0 + lane; e <= e1; e += 32)
            {
              long long b = b0, node = e - b0 * g.ld;
              while (node >= g.ld) // more than one block per chunk only when ld < LIVE_CHUNK
                {
                  node -= g.ld;
                  ++b;
                }
              any = any || (node < g.N && ((node_mask[node] >> (b - 2)) & 1u) != 0u);
            }
        if (__any_sync(0xffffffffu, any) && lane == 0)
          atomicOr(&s_bits, 1u << k);
      }
    __syncthreads();
    if (threadIdx.x == 0 && word < n_words)
      live[word] = s_bits;
  }

  // u <- u_old on the grain DoFs no relevant cell reaches (node_mask bit clear).
  __global__ void __launch_bounds__(256) cut_off_freeze_kernel(const Grid g, int G, const uint16_t *__restrict__ node_mask,
                                                               double *__restrict__ u, const double *__restrict__ u_old)
  {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.N)
      return;
    const unsigned m = node_mask[n];
    for (int b = 0; b < G; ++b)
      if (((m >> b) & 1u) == 0u)
        u[(2 + b) * g.ld + n] = u_old[(2 + b) * g.ld + n];
  }

  static long long cell_count(const Ctx *c) { return (long long)c->grid.n[0] * c->grid.n[1] * c->grid.n[2]; }
  static long long live_words(const Ctx *c)
  {
    const long long chunks = ((long long)c->C * c->ld + LIVE_CHUNK - 1) / LIVE_CHUNK;
    return (chunks + 31) / 32;
  }

  static int allocate_cut(Ctx *c)
  {
    const long long nt = c->grid.n_tiles;
    c->n_cells         = cell_count(c);
    cudaError_t e      = cudaSuccess;
    if ((e = cudaMalloc(&c->mask, sizeof(uint16_t) * (size_t)c->n_cells)) != cudaSuccess ||
        (e = cudaMalloc(&c->cut_tiles, sizeof(int) * (size_t)nt)) != cudaSuccess ||
        (e = cudaMalloc(&c->cut_grains, sizeof(unsigned long long) * (size_t)nt)) != cudaSuccess ||
        (e = cudaMalloc(&c->cut_union, sizeof(uint16_t) * (size_t)nt)) != cudaSuccess ||
        (e = cudaMalloc(&c->tile_union, sizeof(uint16_t) * (size_t)nt)) != cudaSuccess ||
        (e = cudaMalloc(&c->cut_range, sizeof(int) * (SINT_MAX_GRAINS + 2))) != cudaSuccess ||
        (e = cudaMalloc(&c->cut_count, sizeof(unsigned) * (SINT_MAX_GRAINS + 1))) != cudaSuccess ||
        (e = cudaMalloc(&c->node_mask, sizeof(uint16_t) * (size_t)c->grid.N)) != cudaSuccess ||
        (e = cudaMalloc(&c->live, sizeof(uint32_t) * (size_t)live_words(c))) != cudaSuccess)
      {
        cudaFree(c->mask);
        cudaFree(c->cut_tiles);
        cudaFree(c->cut_grains);
        cudaFree(c->cut_union);
        cudaFree(c->tile_union);
        cudaFree(c->cut_range);
        cudaFree(c->cut_count);
        cudaFree(c->node_mask);
        cudaFree(c->live);
        c->mask = nullptr, c->cut_tiles = nullptr, c->cut_grains = nullptr, c->cut_union = nullptr;
        c->tile_union = nullptr, c->cut_range = nullptr, c->cut_count = nullptr, c->node_mask = nullptr;
        c->live = nullptr;
        return cuda_fail(e, "sint_set_component_mask: allocation");
      }
    c->cut_view.cell_mask   = c->mask;
    c->cut_view.tiles       = c->cut_tiles;
    c->cut_view.tile_grains = c->cut_grains;
    c->cut_view.tile_mask   = c->cut_union;
    c->cut_view.range       = c->cut_range;
    c->cut_view.c_all       = c->C;
    return SINT_OK;
  }
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
    if (int rc = allocate_cut(c))
      return rc;
  const long long nb = (c->n_cells + 255) / 256, nbt = (c->grid.n_tiles + 255) / 256;
  grain_mask_kernel<<<dim3((unsigned)nb), 256, 0, stream>>>(c->grid, c->G, u, tol, c->mask);
  if ((e = cudaMemsetAsync(c->cut_count, 0, sizeof(unsigned) * (SINT_MAX_GRAINS + 1), stream)) == cudaSuccess)
    {
      tile_union_kernel<<<dim3((unsigned)nbt), 256, 0, stream>>>(c->grid, c->mask, c->tile_union, c->cut_count);
      class_scan_kernel<<<1, 32, 0, stream>>>(c->G, c->cut_count, c->cut_range);
      class_scatter_kernel<<<dim3((unsigned)nbt), 256, 0, stream>>>(c->grid.n_tiles, c->tile_union, c->cut_count,
                                                                    c->cut_tiles, c->cut_grains, c->cut_union);
      const long long nbn = (c->grid.N + 255) / 256, nw = live_words(c);
      node_mask_kernel<<<dim3((unsigned)nbn), 256, 0, stream>>>(c->grid, c->mask, c->node_mask);
      live_chunk_kernel<<<dim3((unsigned)nw), 1024, 0, stream>>>(c->grid, c->C, c->node_mask, c->live, nw);
      count_launches(6);
      e = cudaGetLastError();
    }
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_set_component_mask");
  c->cut     = true;
  c->cut_tol = tol;
  return SINT_OK;
}

int sint_cut_off_freeze(sint_ctx *c, double *u, const double *u_old, sint_stream_t stream)
{
  if (!c || !u || !u_old)
    {
      set_error("sint_cut_off_freeze: null argument");
      return SINT_ERR_ARG;
    }
  if (!c->cut)
    {
      set_error("sint_cut_off_freeze: no grain cut-off set");
      return SINT_ERR_NOT_READY;
    }
  cut_off_freeze_kernel<<<dim3((unsigned)((c->grid.N + 255) / 256)), 256, 0, stream>>>(c->grid, c->G, c->node_mask,
                                                                                       u, u_old);
  count_launches(1);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_cut_off_freeze");
}

int sint_set_cut_off_skip_zero_chunks(sint_ctx *c, int on)
{
  if (!c)
    {
      set_error("null context");
      return SINT_ERR_ARG;
    }
  c->skip_zeros = on != 0;
  return SINT_OK;
}

int sint_set_preconditioner_cut_off(sint_ctx *c, int on)
{
  if (!c)
    {
      set_error("null context");
      return SINT_ERR_ARG;
    }
  c->pc_cut = on != 0;
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
