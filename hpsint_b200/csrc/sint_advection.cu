// Advection (rigid-body motion of the grains): the per-cell segment table and
// the per-segment velocities the residual and J v kernels read
// (AdvectionMechanism, sintering/advection.h:297-520; the terms themselves are
// in the cell kernels).
#include <cmath>
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

  // ---------------------------------------------------------------------
  // The advection mechanism: forces, torques and volumes of the grain
  // segments from the state (AdvectionOperatorGeneric::do_evaluate_forces,
  // sintering/operator_advection.h:131-373), then the velocity table
  // (AdvectionMechanism, advection.h:330-352).
  //
  // Determinism: the (order parameter, cell) pairs with a segment are sorted
  // by segment once per table (a stable counting sort, items in ascending
  // (b, cell) order within each segment); the force kernel sums fixed tiles
  // of that list, every piece of a segment inside a tile in a fixed order,
  // and a per-segment pass adds the pieces in tile order.  The piece of
  // segment s in tile k is stored at slot s + k: the list is sorted by
  // segment, so no two pieces share a slot.

  constexpr int ADV_TILE  = 512;  // sorted items per block of the force kernel
  constexpr int ADV_NC    = 7;    // volume, force (3), torque (3) per item
  constexpr int ADV_HIST  = 1 << 26; // bound on the count-table entries of the sort

  // Counting sort, pass 1: block r counts the items of its range per segment.
  __global__ void adv_count_kernel(const int *__restrict__ ids, long long n_items, long long range, int S,
                                   int *__restrict__ hist)
  {
    const long long i0 = blockIdx.x * range, i1 = min(n_items, i0 + range);
    for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x)
      {
        const int s = ids[i];
        if (s >= 0)
          atomicAdd(&hist[(long long)blockIdx.x * S + s], 1);
      }
  }

  // Pass 2: per segment, the exclusive prefix over the blocks (in place) and
  // the segment's total.
  __global__ void adv_row_scan_kernel(int nb, int S, int *__restrict__ hist, long long *__restrict__ total)
  {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S)
      return;
    long long run = 0;
    for (int b = 0; b < nb; ++b)
      {
        const int c                  = hist[(long long)b * S + s];
        hist[(long long)b * S + s] = int(run);
        run += c;
      }
    total[s] = run;
  }

  // Pass 3: exclusive scan of the segment totals (one block): off[0..S].
  __global__ void adv_offsets_kernel(int S, const long long *__restrict__ total, long long *__restrict__ off)
  {
    __shared__ long long part[1024];
    const int            per = (S + 1023) / 1024;
    const int            s0 = threadIdx.x * per, s1 = min(S, s0 + per);
    long long            sum = 0;
    for (int s = s0; s < s1; ++s)
      sum += total[s];
    part[threadIdx.x] = sum;
    __syncthreads();
    if (threadIdx.x == 0)
      {
        long long run = 0;
        for (int t = 0; t < 1024; ++t)
          {
            const long long v = part[t];
            part[t]           = run;
            run += v;
          }
        off[S] = run;
      }
    __syncthreads();
    long long run = part[threadIdx.x];
    for (int s = s0; s < s1; ++s)
      {
        off[s] = run;
        run += total[s];
      }
  }

  // Pass 4: one warp per block places the block's items in order, 32 at a
  // time; the block's count row serves as its cursors.
  __global__ void adv_place_kernel(const int *__restrict__ ids, long long n_items, long long range, int S,
                                   const long long *__restrict__ off, int *__restrict__ hist,
                                   unsigned *__restrict__ items)
  {
    const long long i0 = blockIdx.x * range, i1 = min(n_items, i0 + range);
    const int       lane = threadIdx.x;
    int            *cur  = hist + (long long)blockIdx.x * S;
    for (long long base = i0; base < i1; base += 32)
      {
        const long long i     = base + lane;
        const int       s     = i < i1 ? ids[i] : -1;
        const unsigned  peers = __match_any_sync(0xffffffffu, s);
        const int       rank  = __popc(peers & ((1u << lane) - 1u));
        const int       lead  = __ffs(peers) - 1;
        long long       pos   = 0;
        if (s >= 0 && lane == lead)
          {
            pos = off[s] + cur[s];
            cur[s] += __popc(peers);
          }
        pos = __shfl_sync(0xffffffffu, pos, lead);
        if (s >= 0)
          items[pos + rank] = unsigned(i);
      }
  }

  // Value and gradient of a Q1 field at Gauss point q from its nodal values.
  template <int DIM>
  __device__ __forceinline__ void adv_eval(const double (&u)[1 << DIM], int q, const double (&ih)[3], double &v,
                                           double (&gr)[3])
  {
    const double g0 = 0.5 - 0.5 / sqrt(3.0), g1 = 0.5 + 0.5 / sqrt(3.0);
    double       x[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      x[d] = ((q >> d) & 1) ? g1 : g0;
    v = 0.0;
    gr[0] = gr[1] = gr[2] = 0.0;
#pragma unroll
    for (int l = 0; l < (1 << DIM); ++l)
      {
        double sh[3], ds[3];
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          {
            const bool up = (l >> d) & 1;
            sh[d]         = up ? x[d] : 1.0 - x[d];
            ds[d]         = up ? ih[d] : -ih[d];
          }
        double w = 1.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          w *= sh[d];
        v += w * u[l];
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          {
            double gd = ds[d];
#pragma unroll
            for (int e = 0; e < DIM; ++e)
              if (e != d)
                gd *= sh[e];
            gr[d] += gd * u[l];
          }
      }
  }

  // Nodal values of cell (i, j, k); on a periodic mesh the slaves read
  // their masters, as the operator does (iterates of a Newton solve keep
  // stale slave entries until the solution is distributed).
  template <int DIM>
  __device__ __forceinline__ void adv_nodes(const double *__restrict__ u, const Grid &g, int i, int j, int k,
                                            double (&out)[1 << DIM])
  {
#pragma unroll
    for (int l = 0; l < (1 << DIM); ++l)
      {
        int n[3] = {i + (l & 1), j + ((l >> 1) & 1), DIM == 3 ? k + ((l >> 2) & 1) : 0};
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (((g.periodic >> d) & 1) && n[d] == g.n[d])
            n[d] = 0;
        out[l] = u[node_index(g, n[0], n[1], n[2])];
      }
  }

  struct AdvForceParams
  {
    double k, cgb, ceq, smoothening;
  };

  // Volume, force and torque of item (b, cell) over the cell's points.
  template <int DIM>
  __device__ void adv_item(const Grid &g, int G, const double *__restrict__ u, const uint16_t *__restrict__ mask,
                           const double *__restrict__ origin, const double *__restrict__ center, int b, long long cell,
                           const AdvForceParams &prm, double (&o)[ADV_NC])
  {
    constexpr int NQ = 1 << DIM;
#pragma unroll
    for (int e = 0; e < ADV_NC; ++e)
      o[e] = 0.0;
    const unsigned m = mask ? mask[cell] : 0xffffu;
    if (((m >> b) & 1u) == 0u)
      return;
    const int    i = int(cell % g.n[0]), j = int((cell / g.n[0]) % g.n[1]), k = int(cell / ((long long)g.n[0] * g.n[1]));
    const double ih[3] = {1.0 / g.h[0], 1.0 / g.h[1], 1.0 / g.h[2]};
    double       jxw   = 1.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      jxw *= 0.5 * g.h[d];
    double cn[NQ], en[NQ];
    adv_nodes<DIM>(u, g, i, j, k, cn);
    adv_nodes<DIM>(u + (2 + b) * g.ld, g, i, j, k, en);
    double cq[NQ], eq[NQ], geq[NQ][3];
#pragma unroll
    for (int q = 0; q < NQ; ++q)
      {
        double gc[3];
        adv_eval<DIM>(cn, q, ih, cq[q], gc);
        adv_eval<DIM>(en, q, ih, eq[q], geq[q]);
        o[0] += eq[q] * jxw;
      }
    const double g0 = 0.5 - 0.5 / sqrt(3.0), g1 = 0.5 + 0.5 / sqrt(3.0);
    const int    co[3] = {i, j, k};
    for (int jg = 0; jg < G; ++jg)
      {
        if (jg == b || ((m >> jg) & 1u) == 0u)
          continue;
        double fn[NQ];
        adv_nodes<DIM>(u + (2 + jg) * g.ld, g, i, j, k, fn);
#pragma unroll
        for (int q = 0; q < NQ; ++q)
          {
            double ej, gej[3];
            adv_eval<DIM>(fn, q, ih, ej, gej);
            double f = eq[q] * ej;
            if (prm.cgb > 0.0)
              f = prm.smoothening > 0.0 ? 1.0 / (1.0 + exp(-prm.smoothening * (f - prm.cgb)))
                                        : (f > prm.cgb ? 1.0 : 0.0);
            else
              f *= 4.0;
            const double w = prm.k * (cq[q] - prm.ceq) * f * jxw;
            double       dF[3] = {0.0, 0.0, 0.0}, r[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int d = 0; d < DIM; ++d)
              {
                dF[d] = (geq[q][d] - gej[d]) * w;
                r[d]  = origin[d] + (co[d] + (((q >> d) & 1) ? g1 : g0)) * g.h[d] - center[d];
                o[1 + d] += dF[d];
              }
            if constexpr (DIM == 3)
              {
                o[4] += r[1] * dF[2] - r[2] * dF[1];
                o[5] += r[2] * dF[0] - r[0] * dF[2];
                o[6] += r[0] * dF[1] - r[1] * dF[0];
              }
            else
              o[3] += r[1] * dF[0] - r[0] * dF[1]; // hpsint's 2D cross product (tensor.h:62-66)
          }
      }
  }

  // Force kernel: block k sums the pieces of tile k of the sorted item list
  // into slots[(s + k) * ADV_NC ..].
  template <int DIM>
  __global__ void __launch_bounds__(256) adv_force_kernel(Grid g, int G, const double *__restrict__ u,
                                                          const uint16_t *__restrict__ mask, AdvData a,
                                                          const double *__restrict__ centers,
                                                          const unsigned *__restrict__ items, long long n_valid,
                                                          AdvForceParams prm, double *__restrict__ slots)
  {
    __shared__ double sc[ADV_TILE * ADV_NC];
    __shared__ int    key[ADV_TILE];
    __shared__ int    starts[ADV_TILE];
    __shared__ int    n_starts;
    const long long   n_cells = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long   p0      = (long long)blockIdx.x * ADV_TILE;
    const int         len     = int(min((long long)ADV_TILE, n_valid - p0));
    if (threadIdx.x == 0)
      n_starts = 0;
    for (int t = threadIdx.x; t < ADV_TILE; t += blockDim.x)
      {
        double o[ADV_NC];
        int    s = -1;
        if (t < len)
          {
            const unsigned  it   = items[p0 + t];
            const int       b    = int(it / n_cells);
            const long long cell = it - (long long)b * n_cells;
            s                    = a.cell_segments[it];
            adv_item<DIM>(g, G, u, mask, a.origin, centers + 3 * (long long)s, b, cell, prm, o);
          }
        else
#pragma unroll
          for (int e = 0; e < ADV_NC; ++e)
            o[e] = 0.0;
        key[t] = s;
#pragma unroll
        for (int e = 0; e < ADV_NC; ++e)
          sc[t * ADV_NC + e] = o[e];
      }
    __syncthreads();
    for (int t = threadIdx.x; t < len; t += blockDim.x)
      if (t == 0 || key[t] != key[t - 1])
        starts[atomicAdd(&n_starts, 1)] = t;
    __syncthreads();
    // one warp per piece: a fixed lane-strided sum and a fixed shuffle tree
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int r = warp; r < n_starts; r += nw)
      {
        const int t0 = starts[r], s = key[t0];
        int       t1 = t0 + 1;
        while (t1 < len)
          {
            const int  t     = t1 + lane;
            const bool other = t >= len || key[t] != s;
            const unsigned bal = __ballot_sync(0xffffffffu, other);
            if (bal)
              {
                t1 += __ffs(bal) - 1;
                break;
              }
            t1 += 32;
          }
        t1 = min(t1, len);
#pragma unroll
        for (int e = 0; e < ADV_NC; ++e)
          {
            double v = 0.0;
            for (int t = t0 + lane; t < t1; t += 32)
              v += sc[t * ADV_NC + e];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
              v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0)
              slots[((long long)s + blockIdx.x) * ADV_NC + e] = v;
          }
      }
  }

  // Per segment: the pieces in tile order, then the velocity table row.
  __global__ void adv_segment_kernel(int dim, int S, const long long *__restrict__ off,
                                     const double *__restrict__ slots, const double *__restrict__ centers, double mt,
                                     double mr, double *__restrict__ vft, double *__restrict__ table)
  {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S)
      return;
    double sum[ADV_NC];
#pragma unroll
    for (int e = 0; e < ADV_NC; ++e)
      sum[e] = 0.0;
    if (off[s + 1] > off[s])
      {
        const long long k0 = off[s] / ADV_TILE, k1 = (off[s + 1] - 1) / ADV_TILE;
        for (long long k = k0; k <= k1; ++k)
#pragma unroll
          for (int e = 0; e < ADV_NC; ++e)
            sum[e] += slots[((long long)s + k) * ADV_NC + e];
      }
    const int nt = dim == 3 ? 3 : 1, nc = 1 + dim + nt;
    // sum[] holds volume, force[0..2], torque[0..2] (2D: force in 1..2, torque in 3)
    for (int e = 0; e < nc; ++e)
      vft[(long long)s * nc + e] = sum[e];
    double *o = table + 9 * (long long)s;
    for (int e = 0; e < 9; ++e)
      o[e] = 0.0;
    for (int e = 0; e < 3; ++e)
      o[6 + e] = centers[3 * (long long)s + e];
    if (sum[0] > 0.0)
      {
        for (int e = 0; e < dim; ++e)
          o[e] = mt * sum[1 + e] / sum[0];
        if (dim == 3)
          for (int e = 0; e < 3; ++e)
            o[3 + e] = mr * sum[4 + e] / sum[0];
        else
          o[5] = mr * sum[3] / sum[0];
      }
  }

  // CFLChecker::check_courant (sintering/cfl_checker.h:62-128): flags any
  // (cell, relevant grain with a velocity, point) with |v| dt >= diameter.
  __global__ void adv_courant_kernel(Grid g, int G, const uint16_t *__restrict__ mask, AdvData a, double dt,
                                     double diam, unsigned *__restrict__ bad)
  {
    const long long n_cells = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long it      = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (it >= n_cells * G)
      return;
    const int       b    = int(it / n_cells);
    const long long cell = it - b * n_cells;
    if (mask && ((mask[cell] >> b) & 1u) == 0u)
      return;
    const int s = a.cell_segments[it];
    if (s < 0 || s >= a.n_segments)
      return;
    const int     co[3] = {int(cell % g.n[0]), int((cell / g.n[0]) % g.n[1]), int(cell / ((long long)g.n[0] * g.n[1]))};
    const double *d     = a.segments + 9 * (long long)s;
    const double  gp[2] = {0.5 - 0.5 / sqrt(3.0), 0.5 + 0.5 / sqrt(3.0)};
    for (int q = 0; q < (1 << g.dim); ++q)
      {
        double r[3] = {0.0, 0.0, 0.0};
        for (int e = 0; e < g.dim; ++e)
          r[e] = a.origin[e] + (co[e] + gp[(q >> e) & 1]) * g.h[e] - d[6 + e];
        const double v0 = d[0] + d[4] * r[2] - d[5] * r[1];
        const double v1 = d[1] + d[5] * r[0] - d[3] * r[2];
        const double v2 = g.dim == 3 ? d[2] + d[3] * r[1] - d[4] * r[0] : 0.0;
        if (!(sqrt(v0 * v0 + v1 * v1 + v2 * v2) * dt < diam))
          {
            atomicOr(bad, 1u);
            return;
          }
      }
  }

  // Velocity table with zero velocities at the given centers.
  __global__ void adv_init_table_kernel(int S, const double *__restrict__ centers, double *__restrict__ table)
  {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S)
      return;
    for (int e = 0; e < 9; ++e)
      table[9 * (long long)s + e] = e < 6 ? 0.0 : centers[3 * (long long)s + e - 6];
  }

  template <typename T>
  static int grow(T *&ptr, long long &cap, long long need, const char *what)
  {
    if (need <= cap)
      return SINT_OK;
    cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    if (const cudaError_t e = cudaMalloc(&ptr, sizeof(T) * (size_t)(need > 0 ? need : 1)))
      {
        ptr = nullptr;
        return cuda_fail(e, what);
      }
    cap = need;
    return SINT_OK;
  }

  // Copies the per-cell segment ids into the context and checks them against
  // [-1, n_segments); synchronises the stream.
  static int load_cells(Ctx *c, const int *cell_segments, int n_segments, cudaStream_t s, const char *what)
  {
    const long long n_cells = (long long)c->grid.n[0] * c->grid.n[1] * c->grid.n[2], n_ids = n_cells * c->G;
    long long       cap     = c->adv_cells ? n_ids : 0;
    if (int rc = grow(c->adv_cells, cap, n_ids, what))
      return rc;
    long long one = c->adv_error ? 1 : 0;
    if (int rc = grow(c->adv_error, one, 1, what))
      return rc;
    unsigned    bad = 0;
    cudaError_t e   = cudaSuccess;
    if ((e = cudaMemcpyAsync(c->adv_cells, cell_segments, sizeof(int) * (size_t)n_ids, cudaMemcpyDeviceToDevice,
                             s)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->adv_error, 0, sizeof(unsigned), s)) != cudaSuccess)
      return cuda_fail(e, what);
    advection_check_kernel<<<dim3((unsigned)((n_ids + 255) / 256)), 256, 0, s>>>(c->adv_cells, n_ids, n_segments,
                                                                                  c->adv_error);
    count_launches(1);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(&bad, c->adv_error, sizeof(unsigned), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return cuda_fail(e, what);
    if (bad)
      {
        set_error(std::string(what) + ": " + std::to_string(bad) + " segment ids outside [-1, n_segments)");
        return SINT_ERR_ARG;
      }
    return SINT_OK;
  }

  static void set_view(Ctx *c, int n_segments)
  {
    c->adv_view.cell_segments = c->adv_cells;
    c->adv_view.segments      = c->adv_segments;
    c->adv_view.n_segments    = n_segments;
    for (int d = 0; d < 3; ++d)
      c->adv_view.origin[d] = c->mesh.origin[d];
  }

  // Forces of the state u and the velocity table from them (the advection
  // mechanism's update before a residual evaluation).
  int advection_update(Ctx *c, const double *u, cudaStream_t s)
  {
    const int S = c->adv_view.n_segments;
    if (S == 0)
      return SINT_OK;
    const AdvForceParams prm{c->adv_prm.k, c->adv_prm.cgb, c->adv_prm.ceq, c->adv_prm.smoothening};
    const long long      nt = (c->adv_n_valid + ADV_TILE - 1) / ADV_TILE;
    if (nt > 0)
      {
        if (c->grid.dim == 3)
          adv_force_kernel<3><<<dim3((unsigned)nt), 256, 0, s>>>(c->grid, c->G, u, active_mask(c), c->adv_view,
                                                                 c->adv_centers, c->adv_items, c->adv_n_valid, prm,
                                                                 c->adv_slots);
        else
          adv_force_kernel<2><<<dim3((unsigned)nt), 256, 0, s>>>(c->grid, c->G, u, active_mask(c), c->adv_view,
                                                                 c->adv_centers, c->adv_items, c->adv_n_valid, prm,
                                                                 c->adv_slots);
        count_launches(1);
      }
    adv_segment_kernel<<<dim3((unsigned)((S + 127) / 128)), 128, 0, s>>>(c->grid.dim, S, c->adv_off, c->adv_slots,
                                                                       c->adv_centers, c->adv_prm.mt, c->adv_prm.mr,
                                                                       c->adv_vft, c->adv_segments);
    count_launches(1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "advection forces");
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
  c->adv      = false; // until the new table is in place
  c->adv_mech = false;
  if (!cell_segments)
    return SINT_OK;
  if (n_segments < 0 || (n_segments > 0 && !segments))
    {
      set_error("sint_set_advection: n_segments must be >= 0 and segments a device pointer");
      return SINT_ERR_ARG;
    }
  if (int rc = load_cells(c, cell_segments, n_segments, stream, "sint_set_advection"))
    return rc;
  if (int rc = grow(c->adv_segments, c->adv_seg_cap, 9ll * n_segments, "sint_set_advection: allocation"))
    return rc;
  if (n_segments > 0)
    if (const cudaError_t e = cudaMemcpyAsync(c->adv_segments, segments, sizeof(double) * 9 * (size_t)n_segments,
                                              cudaMemcpyDeviceToDevice, stream))
      return cuda_fail(e, "sint_set_advection: copy");
  set_view(c, n_segments);
  c->adv = true;
  return SINT_OK;
}

int sint_set_advection_mechanism(sint_ctx *c, const int32_t *cell_segments, const double *centers, int n_segments,
                                 const sint_advection_params *prm, sint_stream_t stream)
{
  if (!c)
    {
      set_error("null context");
      return SINT_ERR_ARG;
    }
  c->adv      = false;
  c->adv_mech = false;
  if (!cell_segments)
    return SINT_OK;
  if (!prm || n_segments < 0 || (n_segments > 0 && !centers))
    {
      set_error("sint_set_advection_mechanism: parameters, n_segments >= 0 and the centers are required");
      return SINT_ERR_ARG;
    }
  const char     *what    = "sint_set_advection_mechanism";
  const long long n_cells = (long long)c->grid.n[0] * c->grid.n[1] * c->grid.n[2], n_items = n_cells * c->G;
  if (n_items >= (1ll << 32))
    {
      set_error("sint_set_advection_mechanism: n_grains x n_cells must stay below 2^32");
      return SINT_ERR_ARG;
    }
  if (int rc = load_cells(c, cell_segments, n_segments, stream, what))
    return rc;
  const int S  = n_segments;
  const int nc = c->grid.dim == 3 ? 7 : 4;
  if (int rc = grow(c->adv_segments, c->adv_seg_cap, 9ll * S, what))
    return rc;
  if (int rc = grow(c->adv_centers, c->adv_cen_cap, 3ll * S, what))
    return rc;
  if (int rc = grow(c->adv_vft, c->adv_vft_cap, (long long)nc * S, what))
    return rc;
  if (int rc = grow(c->adv_off, c->adv_off_cap, 2ll * S + 1, what)) // offsets (S + 1), then totals (S)
    return rc;
  if (int rc = grow(c->adv_items, c->adv_items_cap, n_items, what))
    return rc;
  cudaError_t e = cudaSuccess;
  if (S > 0)
    {
      if ((e = cudaMemcpyAsync(c->adv_centers, centers, sizeof(double) * 3 * (size_t)S, cudaMemcpyDeviceToDevice,
                               stream)) != cudaSuccess)
        return cuda_fail(e, what);
      adv_init_table_kernel<<<dim3((unsigned)((S + 127) / 128)), 128, 0, stream>>>(S, c->adv_centers,
                                                                                   c->adv_segments);
      count_launches(1);
    }
  // stable counting sort of the items by segment
  long long n_valid = 0;
  if (S > 0)
    {
      long long nb = (n_items + 8191) / 8192;
      nb           = nb < 1 ? 1 : (nb > 4096 ? 4096 : nb);
      while (nb > 1 && nb * S > ADV_HIST)
        nb /= 2;
      const long long range = (n_items + nb - 1) / nb;
      int            *hist  = nullptr;
      if ((e = cudaMalloc(&hist, sizeof(int) * (size_t)(nb * S))) != cudaSuccess)
        return cuda_fail(e, what);
      long long *off = c->adv_off, *total = c->adv_off + S + 1;
      if ((e = cudaMemsetAsync(hist, 0, sizeof(int) * (size_t)(nb * S), stream)) == cudaSuccess)
        {
          adv_count_kernel<<<dim3((unsigned)nb), 256, 0, stream>>>(c->adv_cells, n_items, range, S, hist);
          adv_row_scan_kernel<<<dim3((unsigned)((S + 127) / 128)), 128, 0, stream>>>(int(nb), S, hist, total);
          adv_offsets_kernel<<<1, 1024, 0, stream>>>(S, total, off);
          adv_place_kernel<<<dim3((unsigned)nb), 32, 0, stream>>>(c->adv_cells, n_items, range, S, off, hist,
                                                                   c->adv_items);
          count_launches(4);
          if ((e = cudaGetLastError()) == cudaSuccess &&
              (e = cudaMemcpyAsync(&n_valid, off + S, sizeof(long long), cudaMemcpyDeviceToHost, stream)) ==
                cudaSuccess)
            e = cudaStreamSynchronize(stream);
        }
      cudaFree(hist);
      if (e != cudaSuccess)
        return cuda_fail(e, what);
    }
  c->adv_n_valid = n_valid;
  const long long n_tiles = (n_valid + ADV_TILE - 1) / ADV_TILE;
  if (int rc = grow(c->adv_slots, c->adv_slots_cap, (long long)ADV_NC * (S + n_tiles), what))
    return rc;
  c->adv_prm = *prm;
  set_view(c, S);
  c->adv      = true;
  c->adv_mech = true;
  return SINT_OK;
}

int sint_advection_forces(sint_ctx *c, const double *u, double *vft, sint_stream_t stream)
{
  if (!c || !u)
    {
      set_error("sint_advection_forces: null argument");
      return SINT_ERR_ARG;
    }
  if (!c->adv_mech)
    {
      set_error("sint_advection_forces: no advection mechanism set");
      return SINT_ERR_NOT_READY;
    }
  if (int rc = advection_update(c, u, stream))
    return rc;
  const int S = c->adv_view.n_segments, nc = c->grid.dim == 3 ? 7 : 4;
  if (vft && S > 0)
    if (const cudaError_t e = cudaMemcpyAsync(vft, c->adv_vft, sizeof(double) * (size_t)nc * S,
                                              cudaMemcpyDeviceToDevice, stream))
      return cuda_fail(e, "sint_advection_forces: copy");
  return SINT_OK;
}

int sint_advection_check_courant(sint_ctx *c, double dt, int *ok, sint_stream_t stream)
{
  if (!c || !ok || !(dt >= 0.0))
    {
      set_error("sint_advection_check_courant: null argument or negative dt");
      return SINT_ERR_ARG;
    }
  if (!c->adv)
    {
      set_error("sint_advection_check_courant: no advection set");
      return SINT_ERR_NOT_READY;
    }
  const long long n_items = (long long)c->grid.n[0] * c->grid.n[1] * c->grid.n[2] * c->G;
  double          diam2   = 0.0;
  for (int d = 0; d < c->grid.dim; ++d)
    diam2 += c->grid.h[d] * c->grid.h[d];
  unsigned    bad = 0;
  cudaError_t e   = cudaMemsetAsync(c->adv_error, 0, sizeof(unsigned), stream);
  if (e == cudaSuccess)
    {
      adv_courant_kernel<<<dim3((unsigned)((n_items + 255) / 256)), 256, 0, stream>>>(
        c->grid, c->G, active_mask(c), c->adv_view, dt, std::sqrt(diam2), c->adv_error);
      count_launches(1);
      if ((e = cudaGetLastError()) == cudaSuccess &&
          (e = cudaMemcpyAsync(&bad, c->adv_error, sizeof(unsigned), cudaMemcpyDeviceToHost, stream)) == cudaSuccess)
        e = cudaStreamSynchronize(stream);
    }
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_advection_check_courant");
  *ok = bad ? 0 : 1;
  return SINT_OK;
}
