// Grain-tracker particle detection on the device: the flood fill of one
// order parameter (GrainTracker::run_flooding / detect_local_particle_groups,
// grain_tracker/distributed_stitching.h:41-100, :441-480) as a connected-
// component labelling of the thresholded cells, and the particle properties
// of the spherical representation (compute_particles_info, :264-320;
// compute_particles_radii, :322-360; the particle maxima of run_flooding).
//
// Labelling: union-find over face-neighbour pairs in which a root is only
// ever linked under a smaller cell index, so every component ends with its
// smallest cell as the root whatever the order of the atomic links.
// Particles are numbered by that smallest cell (a scan over the roots in
// lexicographic order), which is the order a lexicographic flood fill
// reaches them.  Properties come from integer moment sums and atomic maxima
// on order-preserving keys, so they do not depend on the thread order either.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "sint_internal.h"
#include "sint_launch.h"

namespace sint
{
  constexpr int SEG_BLOCK = 1024;      // cells per block of the scan
  constexpr int SEG_ACC   = 6;         // accumulators per particle (see seg_acc_kernel)
  constexpr int SEG_LINKS = 1 << 24;   // bound on the retries of one union (never reached)

  __device__ __forceinline__ void cell_coords(const Grid &g, long long c, int &i, int &j, int &k)
  {
    i = int(c % g.n[0]);
    j = int((c / g.n[0]) % g.n[1]);
    k = int(c / ((long long)g.n[0] * g.n[1]));
  }

  __device__ __forceinline__ double cell_max_value(const Grid &g, const double *__restrict__ eta, long long c)
  {
    int i, j, k;
    cell_coords(g, c, i, j, k);
    double mx = eta[node_index(g, i, j, k)];
    for (int l = 1; l < (g.dim == 3 ? 8 : 4); ++l)
      mx = fmax(mx, eta[node_index(g, i + (l & 1), j + ((l >> 1) & 1), k + ((l >> 2) & 1))]);
    return mx;
  }

  // run_flooding's test (distributed_stitching.h:77-79): the largest nodal
  // value of the cell exceeds the threshold.  parent = own index or -1.
  __global__ void __launch_bounds__(256)
    seg_flag_kernel(const Grid g, const double *__restrict__ eta, double thr, int *__restrict__ parent)
  {
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n)
      parent[c] = cell_max_value(g, eta, c) > thr ? int(c) : -1;
  }

  // Root of x; halves the path on the way (parent[x] <= x, so the walk ends).
  __device__ __forceinline__ int seg_find(int *parent, int x)
  {
    int p = parent[x];
    while (p != x)
      {
        const int gp = parent[p];
        if (gp < p)
          parent[x] = gp;
        x = p;
        p = gp;
      }
    return x;
  }

  // Face neighbours in -x, -y, -z (each pair once): link the larger root under
  // the smaller one; a failed compare-and-swap means the root moved: retry.
  __global__ void __launch_bounds__(256) seg_union_kernel(const Grid g, int *parent, int *__restrict__ error)
  {
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || parent[c] < 0)
      return;
    int co[3];
    cell_coords(g, c, co[0], co[1], co[2]);
    const long long stride[3] = {1, g.n[0], (long long)g.n[0] * g.n[1]};
    for (int d = 0; d < g.dim; ++d)
      {
        if (co[d] == 0 || parent[c - stride[d]] < 0)
          continue;
        int a = int(c), b = int(c - stride[d]), it = 0;
        for (; it < SEG_LINKS; ++it)
          {
            a = seg_find(parent, a);
            b = seg_find(parent, b);
            if (a == b)
              break;
            if (a < b)
              {
                const int t = a;
                a           = b;
                b           = t;
              }
            if (atomicCAS(&parent[a], a, b) == a)
              break;
          }
        if (it == SEG_LINKS)
          atomicExch(error, 1);
      }
  }

  // Root of x without writing: once the links are done the forest is fixed,
  // and the only writes left are the final roots of seg_compress_kernel (a
  // halving write there could land after another cell's final root and
  // undo it).
  __device__ __forceinline__ int seg_root(const int *parent, int x)
  {
    int p = parent[x];
    while (p != x)
      {
        x = p;
        p = parent[x];
      }
    return x;
  }

  // Every labelled cell points at its root; block_roots[b] = roots in block b.
  __global__ void __launch_bounds__(SEG_BLOCK)
    seg_compress_kernel(long long n, int *parent, int *__restrict__ block_roots)
  {
    __shared__ int s_count;
    if (threadIdx.x == 0)
      s_count = 0;
    __syncthreads();
    const long long c = (long long)blockIdx.x * SEG_BLOCK + threadIdx.x;
    if (c < n && parent[c] >= 0)
      {
        const int r = seg_root(parent, int(c));
        parent[c]   = r;
        if (r == int(c))
          atomicAdd(&s_count, 1);
      }
    __syncthreads();
    if (threadIdx.x == 0)
      block_roots[blockIdx.x] = s_count;
  }

  // One block: exclusive scan of the per-block root counts (in place), total
  // in block_roots[n_blocks].
  __global__ void __launch_bounds__(1024) seg_scan_blocks_kernel(int n_blocks, int *block_roots)
  {
    __shared__ int s_part[1024];
    const int per = (n_blocks + 1023) / 1024, b0 = threadIdx.x * per;
    int       sum = 0;
    for (int b = b0; b < b0 + per && b < n_blocks; ++b)
      sum += block_roots[b];
    s_part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1)
      {
        const int v = threadIdx.x >= off ? s_part[threadIdx.x - off] : 0;
        __syncthreads();
        s_part[threadIdx.x] += v;
        __syncthreads();
      }
    int run = threadIdx.x == 0 ? 0 : s_part[threadIdx.x - 1];
    for (int b = b0; b < b0 + per && b < n_blocks; ++b)
      {
        const int v    = block_roots[b];
        block_roots[b] = run;
        run += v;
      }
    if (threadIdx.x == 1023)
      block_roots[n_blocks] = s_part[1023];
  }

  // Particle number of every root (its rank among the roots in cell order),
  // written at the root's slot of ids.
  __global__ void __launch_bounds__(SEG_BLOCK)
    seg_rank_kernel(long long n, const int *__restrict__ parent, const int *__restrict__ block_offset,
                    int *__restrict__ ids)
  {
    __shared__ int s_warp[SEG_BLOCK / 32];
    const long long c    = (long long)blockIdx.x * SEG_BLOCK + threadIdx.x;
    const bool      root = c < n && parent[c] == int(c);
    const unsigned  bal  = __ballot_sync(0xffffffffu, root);
    const int       lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
      s_warp[warp] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0)
      {
        int run = 0;
        for (int w = 0; w < SEG_BLOCK / 32; ++w)
          {
            const int v = s_warp[w];
            s_warp[w]   = run;
            run += v;
          }
      }
    __syncthreads();
    if (root)
      ids[c] = block_offset[blockIdx.x] + s_warp[warp] + __popc(bal & ((1u << lane) - 1u));
  }

  __global__ void __launch_bounds__(256)
    seg_label_kernel(long long n, const int *__restrict__ parent, int *__restrict__ ids)
  {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n)
      return;
    const int p = parent[c];
    if (p < 0)
      ids[c] = -1;
    else if (p != int(c))
      ids[c] = ids[p]; // roots keep the rank written before
  }

  // Keys that order like the doubles they encode.
  __host__ __device__ __forceinline__ unsigned long long order_key(unsigned long long bits)
  {
    return (bits >> 63) ? ~bits : (bits | 0x8000000000000000ull);
  }
  __host__ __device__ __forceinline__ unsigned long long order_key_inverse(unsigned long long key)
  {
    return (key >> 63) ? (key & 0x7fffffffffffffffull) : ~key;
  }

  // Per particle p: acc[6p] = cells, acc[6p+1..3] = sums of the cell indices
  // i, j, k, acc[6p+4] = key of the largest nodal value (run_flooding's
  // max_value), acc[6p+5] = radius (pass 2).
  __global__ void __launch_bounds__(256) seg_acc_kernel(const Grid g, const double *__restrict__ eta,
                                                        const int *__restrict__ ids, int n_particles,
                                                        unsigned long long *__restrict__ acc, int *__restrict__ error)
  {
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n)
      return;
    const int p = ids[c];
    if (p < 0)
      return;
    if (p >= n_particles)
      {
        atomicExch(error, 1);
        return;
      }
    int i, j, k;
    cell_coords(g, c, i, j, k);
    unsigned long long *a = acc + (long long)SEG_ACC * p;
    atomicAdd(a + 0, 1ull);
    atomicAdd(a + 1, (unsigned long long)i);
    atomicAdd(a + 2, (unsigned long long)j);
    atomicAdd(a + 3, (unsigned long long)k);
    atomicMax(a + 4, order_key((unsigned long long)__double_as_longlong(cell_max_value(g, eta, c))));
  }

  __host__ __device__ __forceinline__ double seg_center(const unsigned long long *a, int d, double origin,
                                                        double h)
  {
    return origin + h * (double(a[1 + d]) / double(a[0]) + 0.5);
  }

  // compute_particles_radii: max over the cells of |barycenter - center| + diameter / 2.
  __global__ void __launch_bounds__(256)
    seg_radius_kernel(const Grid g, const double o0, const double o1, const double o2, const int *__restrict__ ids,
                      unsigned long long *__restrict__ acc)
  {
    const long long n = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n)
      return;
    const int p = ids[c];
    if (p < 0)
      return;
    int co[3];
    cell_coords(g, c, co[0], co[1], co[2]);
    unsigned long long *a      = acc + (long long)SEG_ACC * p;
    const double        org[3] = {o0, o1, o2};
    double              r2 = 0.0, d2 = 0.0;
    for (int d = 0; d < g.dim; ++d)
      {
        const double x = org[d] + (co[d] + 0.5) * g.h[d], ctr = seg_center(a, d, org[d], g.h[d]);
        r2 += (x - ctr) * (x - ctr);
        d2 += g.h[d] * g.h[d];
      }
    const double r = sqrt(r2) + 0.5 * sqrt(d2);
    atomicMax(a + 5, (unsigned long long)__double_as_longlong(r)); // r >= 0: bits order like values
  }

  static int seg_scratch(Ctx *c, int n_particles)
  {
    const long long n  = (long long)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
    const long long nb = (n + SEG_BLOCK - 1) / SEG_BLOCK;
    cudaError_t     e  = cudaSuccess;
    if (!c->seg_parent)
      {
        if ((e = cudaMalloc(&c->seg_parent, sizeof(int) * (size_t)n)) != cudaSuccess ||
            (e = cudaMalloc(&c->seg_blocks, sizeof(int) * (size_t)(nb + 1))) != cudaSuccess ||
            (e = cudaMalloc(&c->seg_error, sizeof(int))) != cudaSuccess)
          return cuda_fail(e, "grain segments: allocation");
      }
    if (n_particles > c->seg_acc_cap)
      {
        cudaFree(c->seg_acc);
        c->seg_acc     = nullptr;
        c->seg_acc_cap = 0;
        if ((e = cudaMalloc(&c->seg_acc, sizeof(unsigned long long) * SEG_ACC * (size_t)n_particles)) != cudaSuccess)
          return cuda_fail(e, "grain segments: allocation");
        c->seg_acc_cap = n_particles;
      }
    return SINT_OK;
  }
  // Periodicity between particles (tracker.h:1290-1336): for every pair of
  // cells facing each other across a periodic boundary (coordinate n[d] - 1
  // and 0 in direction d) that both belong to particles, the pair of particle
  // ids (smaller first).  Appends to pairs[2 k ..] with a cursor (capacity =
  // the number of such cell pairs, so it never overflows).
  __global__ void seg_periodic_kernel(Grid g, const int *__restrict__ ids, int *__restrict__ pairs,
                                      unsigned *__restrict__ count)
  {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long       base = 0;
    for (int d = 0; d < g.dim; ++d)
      {
        if (!((g.periodic >> d) & 1))
          continue;
        const long long face = (long long)g.n[0] * g.n[1] * g.n[2] / g.n[d];
        if (t >= base + face)
          {
            base += face;
            continue;
          }
        // face cell index f -> coordinates of the other directions
        long long f  = t - base;
        int       co[3];
        for (int e = 0; e < 3; ++e)
          {
            if (e == d)
              continue;
            co[e] = int(f % g.n[e]);
            f /= g.n[e];
          }
        co[d]             = 0;
        const long long c0 = co[0] + (long long)g.n[0] * (co[1] + (long long)g.n[1] * co[2]);
        co[d]             = g.n[d] - 1;
        const long long c1 = co[0] + (long long)g.n[0] * (co[1] + (long long)g.n[1] * co[2]);
        const int       p = ids[c0], q = ids[c1];
        if (p >= 0 && q >= 0)
          {
            const unsigned k = atomicAdd(count, 1u);
            pairs[2 * k]     = min(p, q);
            pairs[2 * k + 1] = max(p, q);
          }
        return;
      }
  }
} // namespace sint

using namespace sint;

int sint_grain_segments(sint_ctx *c, const double *eta, double threshold_lower, int *particle_ids, int *n_particles,
                        sint_stream_t stream)
{
  if (!c || !eta || !particle_ids || !n_particles)
    {
      set_error("sint_grain_segments: null argument");
      return SINT_ERR_ARG;
    }
  if (int rc = seg_scratch(c, 0))
    return rc;
  const long long n  = (long long)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
  const long long nb = (n + SEG_BLOCK - 1) / SEG_BLOCK;
  if (nb > 1024LL * 1024LL)
    {
      set_error("sint_grain_segments: mesh too large");
      return SINT_ERR_ARG;
    }
  const unsigned g256 = (unsigned)((n + 255) / 256);
  cudaError_t    e    = cudaMemsetAsync(c->seg_error, 0, sizeof(int), stream);
  if (e == cudaSuccess)
    {
      seg_flag_kernel<<<g256, 256, 0, stream>>>(c->grid, eta, threshold_lower, c->seg_parent);
      seg_union_kernel<<<g256, 256, 0, stream>>>(c->grid, c->seg_parent, c->seg_error);
      seg_compress_kernel<<<(unsigned)nb, SEG_BLOCK, 0, stream>>>(n, c->seg_parent, c->seg_blocks);
      seg_scan_blocks_kernel<<<1, 1024, 0, stream>>>(int(nb), c->seg_blocks);
      seg_rank_kernel<<<(unsigned)nb, SEG_BLOCK, 0, stream>>>(n, c->seg_parent, c->seg_blocks, particle_ids);
      seg_label_kernel<<<g256, 256, 0, stream>>>(n, c->seg_parent, particle_ids);
      count_launches(6);
      e = cudaGetLastError();
    }
  int h[2] = {0, 0};
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&h[0], c->seg_blocks + nb, sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&h[1], c->seg_error, sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_grain_segments");
  if (h[1])
    {
      set_error("sint_grain_segments: union did not settle");
      return SINT_ERR_CUDA;
    }
  *n_particles = h[0];
  return SINT_OK;
}

int sint_grain_segment_properties(sint_ctx *c, const double *eta, const int *particle_ids, int n_particles,
                                  double *props, sint_stream_t stream)
{
  if (!c || !eta || !particle_ids || (n_particles > 0 && !props) || n_particles < 0)
    {
      set_error("sint_grain_segment_properties: bad argument");
      return SINT_ERR_ARG;
    }
  if (n_particles == 0)
    return SINT_OK;
  if (int rc = seg_scratch(c, n_particles))
    return rc;
  const long long n    = (long long)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
  const unsigned  g256 = (unsigned)((n + 255) / 256);
  const double   *org  = c->mesh.origin;
  cudaError_t     e    = cudaMemsetAsync(c->seg_acc, 0, sizeof(unsigned long long) * SEG_ACC * n_particles, stream);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(c->seg_error, 0, sizeof(int), stream);
  if (e == cudaSuccess)
    {
      seg_acc_kernel<<<g256, 256, 0, stream>>>(c->grid, eta, particle_ids, n_particles, c->seg_acc, c->seg_error);
      seg_radius_kernel<<<g256, 256, 0, stream>>>(c->grid, org[0], org[1], org[2], particle_ids, c->seg_acc);
      count_launches(2);
      e = cudaGetLastError();
    }
  std::vector<unsigned long long> acc((size_t)SEG_ACC * n_particles);
  int                             err = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(acc.data(), c->seg_acc, sizeof(unsigned long long) * acc.size(), cudaMemcpyDeviceToHost,
                        stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&err, c->seg_error, sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_grain_segment_properties");
  if (err)
    {
      set_error("sint_grain_segment_properties: particle id out of range");
      return SINT_ERR_ARG;
    }
  const int dim = c->grid.dim, nf = 3 + dim;
  double    vol = 1.0;
  for (int d = 0; d < dim; ++d)
    vol *= c->grid.h[d];
  for (int p = 0; p < n_particles; ++p)
    {
      const unsigned long long *a = acc.data() + (size_t)SEG_ACC * p;
      double                   *o = props + (size_t)nf * p;
      o[0]                        = double(a[0]) * vol;
      for (int d = 0; d < dim; ++d)
        o[1 + d] = seg_center(a, d, org[d], c->grid.h[d]);
      unsigned long long rb = a[5], mb = order_key_inverse(a[4]);
      double             r, m;
      std::memcpy(&r, &rb, sizeof(double));
      std::memcpy(&m, &mb, sizeof(double));
      o[1 + dim] = r;
      o[2 + dim] = m;
    }
  return SINT_OK;
}

int sint_grain_segment_periodicity(sint_ctx *c, const int *particle_ids, int *pairs, int max_pairs, int *n_pairs,
                                   sint_stream_t stream)
{
  if (!c || !particle_ids || !n_pairs || max_pairs < 0 || (max_pairs > 0 && !pairs))
    {
      set_error("sint_grain_segment_periodicity: bad argument");
      return SINT_ERR_ARG;
    }
  *n_pairs = 0;
  long long cap = 0;
  for (int d = 0; d < c->grid.dim; ++d)
    if ((c->grid.periodic >> d) & 1)
      cap += (long long)c->grid.n[0] * c->grid.n[1] * c->grid.n[2] / c->grid.n[d];
  if (cap == 0)
    return SINT_OK;
  int         *buf   = nullptr;
  unsigned    *count = nullptr;
  cudaError_t  e     = cudaMalloc(&buf, sizeof(int) * 2 * (size_t)cap);
  if (e == cudaSuccess)
    e = cudaMalloc(&count, sizeof(unsigned));
  unsigned         k = 0;
  std::vector<int> host;
  if (e == cudaSuccess)
    e = cudaMemsetAsync(count, 0, sizeof(unsigned), stream);
  if (e == cudaSuccess)
    {
      seg_periodic_kernel<<<(unsigned)((cap + 255) / 256), 256, 0, stream>>>(c->grid, particle_ids, buf, count);
      count_launches(1);
      e = cudaGetLastError();
    }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&k, count, sizeof(unsigned), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(stream);
  if (e == cudaSuccess && k > 0)
    {
      host.resize(2 * (size_t)k);
      e = cudaMemcpy(host.data(), buf, sizeof(int) * host.size(), cudaMemcpyDeviceToHost);
    }
  cudaFree(buf);
  cudaFree(count);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_grain_segment_periodicity");
  // the set of distinct pairs, in increasing order (std::set in the reference)
  std::vector<std::pair<int, int>> uniq;
  uniq.reserve(k);
  for (unsigned i = 0; i < k; ++i)
    uniq.emplace_back(host[2 * i], host[2 * i + 1]);
  std::sort(uniq.begin(), uniq.end());
  uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
  *n_pairs = int(uniq.size());
  if (int(uniq.size()) > max_pairs)
    {
      set_error("sint_grain_segment_periodicity: more pairs than max_pairs (n_pairs holds the count)");
      return SINT_ERR_ARG;
    }
  for (size_t i = 0; i < uniq.size(); ++i)
    {
      pairs[2 * i]     = uniq[i].first;
      pairs[2 * i + 1] = uniq[i].second;
    }
  return SINT_OK;
}
