// C ABI of the sintering operator: context life cycle, operator and
// preconditioner entry points.  See include/hpsint_b200.h for the contract.
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>

#include "sint_internal.h"
#include "sint_kernels.cuh"
#include "sint_launch.h"

namespace sint
{
  static thread_local std::string g_last_error = "";
  static std::atomic<long long>   g_launches{0};

  void set_error(const std::string &msg) { g_last_error = msg; }

  int cuda_fail(cudaError_t e, const char *what)
  {
    set_error(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    return SINT_ERR_CUDA;
  }

  void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

  size_t smem_diag(int dim, int G, bool adv)
  {
    const int C = G + 2;
    // NCOEF = 2 dim^2 + dim + 1 + G (+ G dim velocities) coefficients per point, NOUT = G + 4 outputs
    const int nadv = adv ? G * dim : 0;
    if (dim == 3)
      return (C * Tile<3>::BOXS + (22 + G + nadv) * Tile<3>::THREADS + (G + 4) * Tile<3>::CS) * sizeof(double);
    return (C * Tile<2>::BOXS + (11 + G + nadv) * Tile<2>::THREADS + (G + 4) * Tile<2>::CS) * sizeof(double);
  }

  template <int DIM, typename R>
  cudaError_t launch_combine(int ncomp, const Grid &g, const R *partial, R *dst, const uint16_t *tile_mask,
                             cudaStream_t s, const ResidualHooks *epi)
  {
    const long long nb   = (g.N + 255) / 256;
    const bool      fin  = epi && epi->epilogue;
    const double   *sub  = fin ? epi->subtract : nullptr;
    const double    sc   = fin ? epi->scale : 1.0;
    // the instance for this component count (C = G + 2 <= 14, the
    // preconditioner's G + 4 <= 16): one thread per node; other counts in 2D
    // one thread per (node, component)
    auto go = [&](auto nc) {
      constexpr int NC = decltype(nc)::value;
      const dim3    grid((unsigned)nb, (DIM == 2 && NC == 0) ? (unsigned)ncomp : 1u);
      combine_kernel<DIM, R, NC><<<grid, 256, 0, s>>>(g, ncomp, partial, dst, tile_mask, sub, sc, fin ? 1 : 0);
    };
    switch (ncomp)
      {
#define SINT_NC(K)                                                                                                \
  case K: go(std::integral_constant<int, K>{}); break;
        SINT_NC(2) SINT_NC(3) SINT_NC(4) SINT_NC(5) SINT_NC(6) SINT_NC(7) SINT_NC(8) SINT_NC(9) SINT_NC(10)
        SINT_NC(11) SINT_NC(12) SINT_NC(13) SINT_NC(14) SINT_NC(15) SINT_NC(16)
#undef SINT_NC
        default: go(std::integral_constant<int, 0>{}); break;
      }
    count_launches(1);
    return cudaGetLastError();
  }

  // dst = (dst - sub) * scale over the C blocks (the residual's epilogue hook
  // on periodic meshes, after the slave rows are condensed)
  __global__ void residual_epilogue_kernel(long long N, long long ld, int C, const double *__restrict__ sub,
                                           double scale, double *__restrict__ dst)
  {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N)
      return;
    for (int b = 0; b < C; ++b)
      dst[b * ld + n] = (dst[b * ld + n] - (sub ? sub[b * ld + n] : 0.0)) * scale;
  }
  template cudaError_t launch_combine<2, double>(int, const Grid &, const double *, double *, const uint16_t *,
                                                cudaStream_t, const ResidualHooks *);
  template cudaError_t launch_combine<3, double>(int, const Grid &, const double *, double *, const uint16_t *,
                                                cudaStream_t, const ResidualHooks *);
  template cudaError_t launch_combine<2, float>(int, const Grid &, const float *, float *, const uint16_t *,
                                                cudaStream_t, const ResidualHooks *);
  template cudaError_t launch_combine<3, float>(int, const Grid &, const float *, float *, const uint16_t *,
                                                cudaStream_t, const ResidualHooks *);

  // --- dispatch over (dim, mobility) ---------------------------------------
  template <typename R>
  cudaError_t dispatch_jvp(const Ctx *c, const R *lin, const R *src, R *dst, cudaStream_t s)
  {
    R *part = reinterpret_cast<R *>(c->partial);
    const bool      t   = c->params.tensorial != 0;
    const CutTiles *cut = active_cut(c);
    const AdvData  *adv = active_adv(c);
    cudaError_t e;
    if (c->grid.dim == 3)
      e = t ? launch_jvp<3, true, R>(c->G, c->grid, c->phys, lin, src, dst, part, cut, adv, s)
            : launch_jvp<3, false, R>(c->G, c->grid, c->phys, lin, src, dst, part, cut, adv, s);
    else
      e = t ? launch_jvp<2, true, R>(c->G, c->grid, c->phys, lin, src, dst, part, cut, adv, s)
            : launch_jvp<2, false, R>(c->G, c->grid, c->phys, lin, src, dst, part, cut, adv, s);
    if (e != cudaSuccess)
      return e;
    e = c->grid.dim == 3 ? launch_combine<3, R>(c->C, c->grid, part, dst, active_tile_union(c), s, nullptr)
                         : launch_combine<2, R>(c->C, c->grid, part, dst, active_tile_union(c), s, nullptr);
    if (e != cudaSuccess)
      return e;
    return launch_periodic_condense<R>(c->grid, c->C, dst, src, 0, s);
  }

  template cudaError_t dispatch_jvp<double>(const Ctx *, const double *, const double *, double *, cudaStream_t);
  template cudaError_t dispatch_jvp<float>(const Ctx *, const float *, const float *, float *, cudaStream_t);

  // hooks: the residual's pre/post range operations in device form (nullptr
  // for none).  The epilogue is fused into the stores and the combine step,
  // except on periodic meshes, where it follows the condensation of the slave
  // rows as one extra pass.
  static cudaError_t dispatch_residual(const Ctx *c, int wtd, const double *src, const double *const *hist,
                                       double *dst, cudaStream_t s, const ResidualHooks *hooks = nullptr)
  {
    const bool      t   = c->params.tensorial != 0;
    const CutTiles *cut = active_cut(c);
    const AdvData  *adv = active_adv(c);
    Phys            ph  = c->phys;
    const bool      epi_after = hooks && hooks->epilogue && c->grid.periodic;
    if (hooks)
      {
        ph.hooks = *hooks;
        if (epi_after)
          ph.hooks.epilogue = 0;
      }
    cudaError_t e;
    if (c->grid.dim == 3)
      e = t ? launch_residual<3, true>(c->G, wtd, c->grid, ph, src, hist, dst, c->partial, cut, adv, s)
            : launch_residual<3, false>(c->G, wtd, c->grid, ph, src, hist, dst, c->partial, cut, adv, s);
    else
      e = t ? launch_residual<2, true>(c->G, wtd, c->grid, ph, src, hist, dst, c->partial, cut, adv, s)
            : launch_residual<2, false>(c->G, wtd, c->grid, ph, src, hist, dst, c->partial, cut, adv, s);
    if (e != cudaSuccess)
      return e;
    e = c->grid.dim == 3 ? launch_combine<3, double>(c->C, c->grid, c->partial, dst, active_tile_union(c), s, &ph.hooks)
                         : launch_combine<2, double>(c->C, c->grid, c->partial, dst, active_tile_union(c), s, &ph.hooks);
    if (e != cudaSuccess)
      return e;
    if ((e = launch_periodic_condense<double>(c->grid, c->C, dst, nullptr, 1, s)) != cudaSuccess || !epi_after)
      return e;
    residual_epilogue_kernel<<<dim3((unsigned)((c->N + 255) / 256)), 256, 0, s>>>(c->N, c->ld, c->C, hooks->subtract,
                                                                                   hooks->scale, dst);
    count_launches(1);
    return cudaGetLastError();
  }

  static cudaError_t dispatch_diag(const Ctx *c, double *dst, cudaStream_t s)
  {
    const bool t = c->params.tensorial != 0;
    cudaError_t e;
    const uint16_t *m   = preconditioner_mask(c);
    const AdvData  *adv = active_adv(c);
    if (c->grid.dim == 3)
      e = t ? launch_diag<3, true>(c->G, c->grid, c->phys, c->lin64, dst, c->partial, m, adv, s)
            : launch_diag<3, false>(c->G, c->grid, c->phys, c->lin64, dst, c->partial, m, adv, s);
    else
      e = t ? launch_diag<2, true>(c->G, c->grid, c->phys, c->lin64, dst, c->partial, m, adv, s)
            : launch_diag<2, false>(c->G, c->grid, c->phys, c->lin64, dst, c->partial, m, adv, s);
    if (e != cudaSuccess)
      return e;
    e = c->grid.dim == 3 ? launch_combine<3, double>(c->G + 4, c->grid, c->partial, dst, nullptr, s, nullptr)
                         : launch_combine<2, double>(c->G + 4, c->grid, c->partial, dst, nullptr, s, nullptr);
    if (e != cudaSuccess)
      return e;
    return launch_periodic_condense<double>(c->grid, c->G + 4, dst, nullptr, 2, s);
  }

  // --- preconditioner point kernels ----------------------------------------
  // Inverts the CH 2x2 node blocks and the AC diagonal.
  __global__ void precond_invert_kernel(long long N, long long ld, int G, const double *__restrict__ raw,
                                        double *__restrict__ inv64, float *__restrict__ inv32)
  {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N)
      return;
    const double a = raw[0 * ld + n], b = raw[1 * ld + n], c = raw[2 * ld + n], d = raw[3 * ld + n];
    const double det   = a * d - b * c;
    const double scale = fabs(a * d) + fabs(b * c);
    double       i00, i01, i10, i11;
    if (det != 0.0 && isfinite(det) && fabs(det) > 1e-14 * scale)
      {
        i00 = d / det;
        i01 = -b / det;
        i10 = -c / det;
        i11 = a / det;
      }
    else
      {
        // singular block: fall back to the guarded point inverse
        i00 = fabs(a) > 1.0e-10 ? 1.0 / a : 1.0;
        i11 = fabs(d) > 1.0e-10 ? 1.0 / d : 1.0;
        i01 = i10 = 0.0;
      }
    inv64[0 * ld + n] = i00;
    inv64[1 * ld + n] = i01;
    inv64[2 * ld + n] = i10;
    inv64[3 * ld + n] = i11;
    inv32[0 * ld + n] = float(i00);
    inv32[1 * ld + n] = float(i01);
    inv32[2 * ld + n] = float(i10);
    inv32[3 * ld + n] = float(i11);
    for (int i = 0; i < G; ++i)
      {
        const double di = raw[(4 + i) * ld + n];
        // operator_base.h:386-388
        const double v    = (fabs(di) > 1.0e-10) ? (1.0 / di) : 1.0;
        inv64[(4 + i) * ld + n] = v;
        inv32[(4 + i) * ld + n] = float(v);
      }
  }

  // z = P^-1 r: 2x2 blocks on (c, mu), point-Jacobi on the grains.
  template <typename R>
  __global__ void precond_apply_kernel(long long N, long long ld, int G, const R *__restrict__ inv,
                                       const R *__restrict__ r, R *__restrict__ z)
  {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N)
      return;
    const R rc = r[n], rm = r[ld + n];
    z[n]      = inv[n] * rc + inv[ld + n] * rm;
    z[ld + n] = inv[2 * ld + n] * rc + inv[3 * ld + n] * rm;
    for (int i = 0; i < G; ++i)
      z[(2 + i) * ld + n] = inv[(4 + i) * ld + n] * r[(2 + i) * ld + n];
  }

  __global__ void f64_to_f32_kernel(long long n, const double *__restrict__ x, float *__restrict__ y)
  {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      y[i] = float(x[i]);
  }

  static bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }
} // namespace sint

using namespace sint;

namespace sint
{
  // Validates mesh and parameters and fills the operator description (mesh,
  // grid, point-wise parameters, layout) of `c`; allocates nothing.
  int describe_operator(const sint_mesh *mesh, const sint_params *params, Ctx *c)
  {
    if (mesh->dim != 2 && mesh->dim != 3)
      {
        set_error("sint_create: dim must be 2 or 3");
        return SINT_ERR_ARG;
      }
    if (params->n_grains < 1 || params->n_grains > SINT_MAX_GRAINS)
      {
        set_error("This operation is precompiled for the number of grains in range [1, " +
                  std::to_string(SINT_MAX_GRAINS) + "] but you provided n_grains = " +
                  std::to_string(params->n_grains));
        return SINT_ERR_GRAINS;
      }
    for (int d = 0; d < mesh->dim; ++d)
      if (mesh->n_cells[d] < 1 || !(mesh->h[d] > 0.0) || !std::isfinite(mesh->h[d]))
        {
          set_error("sint_create: every n_cells[d] must be >= 1 and h[d] > 0");
          return SINT_ERR_ARG;
        }

    c->mesh     = *mesh;
    c->params   = *params;
    c->G        = params->n_grains;
    c->C        = params->n_grains + 2;
    Grid &g     = c->grid;
    g.dim       = mesh->dim;
    const int TT[3] = {mesh->dim == 3 ? Tile<3>::TX : Tile<2>::TX, mesh->dim == 3 ? Tile<3>::TY : Tile<2>::TY,
                       mesh->dim == 3 ? Tile<3>::TZ : 1};
    long long N = 1, nt = 1;
    for (int d = 0; d < 3; ++d)
      {
        if (d < mesh->dim)
          {
            g.n[d]  = mesh->n_cells[d];
            g.nn[d] = mesh->n_cells[d] + 1;
            g.nt[d] = (mesh->n_cells[d] + TT[d] - 1) / TT[d];
            g.h[d]  = mesh->h[d];
          }
        else
          {
            g.n[d] = g.nn[d] = g.nt[d] = 1;
            g.h[d]                     = 1.0;
          }
        N *= g.nn[d];
        nt *= g.nt[d];
      }
    g.N       = N;
    g.n_tiles = nt;
    if (nt >= (1ll << 31) || N >= (1ll << 40))
      {
        set_error("mesh too large: at most 2^31 - 1 tiles");
        return SINT_ERR_ARG;
      }
    for (int d = 0; d < 2; ++d)
      {
        make_divisor((unsigned)g.nt[d], g.mdiv[d], g.sdiv[d]);
        make_divisor((unsigned)g.nn[d], g.mnode[d], g.snode[d]);
      }
    // exact Q1 element Laplacian of the uniform cell: K_lm = kx[l xor m], built
    // from the 1D stiffness (1/h)[[1,-1],[-1,1]] and mass (h/6)[[2,1],[1,2]]
    for (int x = 0; x < 8; ++x)
      {
        double k = 0.0;
        if (x < (1 << mesh->dim))
          for (int d = 0; d < mesh->dim; ++d)
            {
              double t = (((x >> d) & 1) ? -1.0 : 1.0) / g.h[d];
              for (int e = 0; e < mesh->dim; ++e)
                if (e != d)
                  t *= ((x >> e) & 1) ? g.h[e] / 6.0 : g.h[e] / 3.0;
              k += t;
            }
        g.kxd[x] = k;
        g.kxf[x] = float(k);
      }
    g.ld      = (N + 31) / 32 * 32;
    c->N      = N;
    c->ld     = g.ld;

    Phys &p = c->phys;
    std::memset(&p, 0, sizeof(p));
    p.A       = params->A;
    p.B       = params->B;
    p.kappa_c = params->kappa_c;
    p.kappa_p = params->kappa_p;
    p.Mvol    = params->Mvol;
    p.Mvap    = params->Mvap;
    p.Msurf   = params->Msurf;
    p.Mgb     = params->Mgb;
    p.L       = params->L;
    set_row_stiffness(g, p.kappa_c, p.kappa_p, p.L);
    p.w0      = 0.0;
    p.w_alg   = 1.0;
    p.order   = 0;
    return SINT_OK;
  }
} // namespace sint

static int check_ctx(const sint_ctx *ctx)
{
  if (!ctx)
    {
      set_error("null context");
      return SINT_ERR_ARG;
    }
  return SINT_OK;
}

static int check_vec(const void *p, const char *name)
{
  if (!p)
    {
      set_error(std::string("null pointer: ") + name);
      return SINT_ERR_ARG;
    }
  if (!aligned16(p))
    {
      set_error(std::string("pointer not 16-byte aligned: ") + name);
      return SINT_ERR_ARG;
    }
  return SINT_OK;
}

extern "C" {

const char *sint_last_error(void) { return g_last_error.c_str(); }

int64_t sint_kernel_launch_count(void) { return g_launches.load(); }

int sint_create(const sint_mesh *mesh, const sint_params *params, sint_ctx **out)
{
  if (!mesh || !params || !out)
    {
      set_error("sint_create: null argument");
      return SINT_ERR_ARG;
    }
  *out = nullptr;
  sint_ctx *c = new sint_ctx();
  if (int rc = describe_operator(mesh, params, c))
    {
      delete c;
      return rc;
    }
  const Grid &g  = c->grid;
  const long long nt = g.n_tiles;
  const int box   = mesh->dim == 3 ? Tile<3>::BOX : Tile<2>::BOX;
  c->partial_bytes = size_t(nt) * size_t(c->G + 4) * size_t(box) * sizeof(double);
  cudaError_t e;
  const size_t vec64 = size_t(c->C) * g.ld * sizeof(double);
  const size_t pcsz  = size_t(c->G + 4) * g.ld;
  if ((e = cudaMalloc(&c->lin64, vec64)) != cudaSuccess || (e = cudaMalloc(&c->lin32, vec64 / 2)) != cudaSuccess ||
      (e = cudaMalloc(&c->partial, c->partial_bytes)) != cudaSuccess ||
      (e = cudaMalloc(&c->pc_raw, pcsz * sizeof(double))) != cudaSuccess ||
      (e = cudaMalloc(&c->pc_inv64, pcsz * sizeof(double))) != cudaSuccess ||
      (e = cudaMalloc(&c->pc_inv32, pcsz * sizeof(float))) != cudaSuccess ||
      (e = cudaMalloc(&c->red, sizeof(double) * ((MAX_MULTIDOT + 1) * NB_RED + RED_TICKETS))) != cudaSuccess)
    {
      const int rc = cuda_fail(e, "sint_create: cudaMalloc");
      sint_destroy(c);
      return rc;
    }
  c->red_ticket = reinterpret_cast<unsigned *>(c->red + (MAX_MULTIDOT + 1) * NB_RED);
  // padding entries are part of every block vector; keep them defined
  if ((e = cudaMemset(c->lin64, 0, vec64)) != cudaSuccess || (e = cudaMemset(c->lin32, 0, vec64 / 2)) != cudaSuccess ||
      (e = cudaMemset(c->pc_inv64, 0, pcsz * sizeof(double))) != cudaSuccess ||
      (e = cudaMemset(c->pc_inv32, 0, pcsz * sizeof(float))) != cudaSuccess ||
      (e = cudaMemset(c->red_ticket, 0, sizeof(double) * RED_TICKETS)) != cudaSuccess)
    {
      const int rc = cuda_fail(e, "sint_create: cudaMemset");
      sint_destroy(c);
      return rc;
    }
  *out = c;
  return SINT_OK;
}

int sint_destroy(sint_ctx *c)
{
  if (!c)
    return SINT_OK;
  cudaDeviceSynchronize();
  free_workspace(c);
  cudaFree(c->lin64);
  cudaFree(c->lin32);
  cudaFree(c->partial);
  cudaFree(c->mask);
  cudaFree(c->cut_tiles);
  cudaFree(c->cut_grains);
  cudaFree(c->cut_union);
  cudaFree(c->tile_union);
  cudaFree(c->cut_range);
  cudaFree(c->cut_count);
  cudaFree(c->node_mask);
  cudaFree(c->live);
  cudaFree(c->seg_parent);
  cudaFree(c->seg_blocks);
  cudaFree(c->seg_acc);
  cudaFree(c->seg_error);
  cudaFree(c->adv_cells);
  cudaFree(c->adv_segments);
  cudaFree(c->adv_error);
  cudaFree(c->adv_centers);
  cudaFree(c->adv_vft);
  cudaFree(c->adv_off);
  cudaFree(c->adv_items);
  cudaFree(c->adv_slots);
  cudaFree(c->ch_A64);
  cudaFree(c->ch_A32);
  cudaFree(c->ch_dinv64);
  cudaFree(c->ch_dinv32);
  cudaFree(c->pc_raw);
  cudaFree(c->pc_inv64);
  cudaFree(c->pc_inv32);
  cudaFree(c->red);
  delete c;
  return SINT_OK;
}

int sint_dof_layout(const sint_ctx *c, int64_t *n_nodes, int *n_components, int64_t *block_stride)
{
  if (int e = check_ctx(c))
    return e;
  if (n_nodes)
    *n_nodes = c->N;
  if (n_components)
    *n_components = c->C;
  if (block_stride)
    *block_stride = c->ld;
  return SINT_OK;
}

int sint_set_time_weights(sint_ctx *c, double w0, const double *w_hist, int order, double w_alg)
{
  if (int e = check_ctx(c))
    return e;
  if (order < 0 || order > 3 || (order > 0 && !w_hist))
    {
      set_error("sint_set_time_weights: order must be in [0, 3] and w_hist non-null when order > 0");
      return SINT_ERR_ARG;
    }
  c->phys.w0    = w0;
  c->phys.w_alg = w_alg;
  c->phys.order = order;
  for (int i = 0; i < 4; ++i)
    c->phys.w_hist[i] = i < order ? w_hist[i] : 0.0;
  return SINT_OK;
}

int sint_set_mobility(sint_ctx *c, double Mvol, double Mvap, double Msurf, double Mgb, double L)
{
  if (int e = check_ctx(c))
    return e;
  c->phys.Mvol  = c->params.Mvol = Mvol;
  c->phys.Mvap  = c->params.Mvap = Mvap;
  c->phys.Msurf = c->params.Msurf = Msurf;
  c->phys.Mgb   = c->params.Mgb = Mgb;
  c->phys.L     = c->params.L = L;
  sint::set_row_stiffness(c->grid, c->phys.kappa_c, c->phys.kappa_p, L);
  return SINT_OK;
}

int sint_set_linearization_point(sint_ctx *c, const double *u, sint_stream_t stream)
{
  if (int e = check_ctx(c))
    return e;
  if (int e = check_vec(u, "u"))
    return e;
  const size_t n = size_t(c->C) * c->ld;
  cudaError_t  e = cudaMemcpyAsync(c->lin64, u, n * sizeof(double), cudaMemcpyDeviceToDevice, stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_set_linearization_point: copy");
  f64_to_f32_kernel<<<dim3(1184), 256, 0, stream>>>((long long)n, c->lin64, c->lin32);
  count_launches(1);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return cuda_fail(e, "sint_set_linearization_point: shadow");
  c->has_lin = true;
  return SINT_OK;
}

int sint_residual_f64(sint_ctx *c, double *dst, const double *src, const double *const *hist,
                      int with_time_derivative, sint_stream_t stream)
{
  if (int e = check_ctx(c))
    return e;
  if (int e = check_vec(dst, "dst"))
    return e;
  if (int e = check_vec(src, "src"))
    return e;
  if (with_time_derivative < 0 || with_time_derivative > 2)
    {
      set_error("sint_residual_f64: with_time_derivative must be 0, 1 or 2");
      return SINT_ERR_ARG;
    }
  if (with_time_derivative == 2)
    {
      if (c->phys.order < 1 || !hist)
        {
          set_error("sint_residual_f64: with_time_derivative == 2 needs time weights of order >= 1 and hist");
          return SINT_ERR_ARG;
        }
      for (int i = 0; i < c->phys.order; ++i)
        if (int e = check_vec(hist[i], "hist[i]"))
          return e;
    }
  // the advection mechanism moves the grains with the forces of this state
  // (ResidualWrapperAdvection::evaluate_for_residual, residual_wrapper.h:58-64)
  if (c->adv_mech)
    if (int rc = advection_update(c, src, stream))
      return rc;
  const cudaError_t e = dispatch_residual(c, with_time_derivative, src, hist, dst, stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_residual_f64");
  return SINT_OK;
}

int sint_residual_f64_hooks(sint_ctx *c, double *dst, const double *src, const double *const *hist,
                            int with_time_derivative, const sint_residual_hooks *hooks, sint_stream_t stream)
{
  if (!hooks)
    return sint_residual_f64(c, dst, src, hist, with_time_derivative, stream);
  if (int e = check_ctx(c))
    return e;
  if (int e = check_vec(dst, "dst"))
    return e;
  if (int e = check_vec(src, "src"))
    return e;
  if ((hooks->perturb && check_vec(hooks->perturb, "hooks->perturb")) ||
      (hooks->subtract && check_vec(hooks->subtract, "hooks->subtract")))
    return SINT_ERR_ARG;
  if (hooks->perturb == dst || (hooks->subtract == dst && hooks->subtract))
    {
      set_error("sint_residual_f64_hooks: dst must not alias the hook vectors");
      return SINT_ERR_ARG;
    }
  if (hooks->perturb && c->adv_mech)
    {
      set_error("sint_residual_f64_hooks: a perturbed evaluation with the advection mechanism is not supported "
                "(its forces would need the perturbed state); evaluate src + a x into a vector first");
      return SINT_ERR_ARG;
    }
  if (with_time_derivative < 0 || with_time_derivative > 2)
    {
      set_error("sint_residual_f64_hooks: with_time_derivative must be 0, 1 or 2");
      return SINT_ERR_ARG;
    }
  if (with_time_derivative == 2)
    {
      if (c->phys.order < 1 || !hist)
        {
          set_error("sint_residual_f64_hooks: with_time_derivative == 2 needs time weights of order >= 1 and hist");
          return SINT_ERR_ARG;
        }
      for (int i = 0; i < c->phys.order; ++i)
        if (int e = check_vec(hist[i], "hist[i]"))
          return e;
    }
  if (c->adv_mech)
    if (int rc = advection_update(c, src, stream))
      return rc;
  ResidualHooks h;
  h.perturb       = hooks->perturb;
  h.perturb_scale = hooks->perturb ? hooks->perturb_scale : 0.0;
  h.subtract      = hooks->subtract;
  h.scale         = hooks->scale;
  h.epilogue      = (hooks->subtract || hooks->scale != 1.0) ? 1 : 0;
  const cudaError_t e = dispatch_residual(c, with_time_derivative, src, hist, dst, stream, &h);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_residual_f64_hooks");
  return SINT_OK;
}

int sint_jvp_f64(sint_ctx *c, double *dst, const double *src, sint_stream_t stream)
{
  if (int e = check_ctx(c))
    return e;
  if (!c->has_lin)
    {
      set_error("sint_jvp_f64: no linearisation point set");
      return SINT_ERR_NOT_READY;
    }
  if (int e = check_vec(dst, "dst"))
    return e;
  if (int e = check_vec(src, "src"))
    return e;
  const cudaError_t e = dispatch_jvp<double>(c, c->lin64, src, dst, stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_jvp_f64");
  return SINT_OK;
}

int sint_jvp_f32(sint_ctx *c, float *dst, const float *src, sint_stream_t stream)
{
  if (int e = check_ctx(c))
    return e;
  if (!c->has_lin)
    {
      set_error("sint_jvp_f32: no linearisation point set");
      return SINT_ERR_NOT_READY;
    }
  if (int e = check_vec(dst, "dst"))
    return e;
  if (int e = check_vec(src, "src"))
    return e;
  const cudaError_t e = dispatch_jvp<float>(c, c->lin32, src, dst, stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_jvp_f32");
  return SINT_OK;
}

int sint_precond_setup(sint_ctx *c, sint_stream_t stream)
{
  if (int e = check_ctx(c))
    return e;
  if (!c->has_lin)
    {
      set_error("sint_precond_setup: no linearisation point set");
      return SINT_ERR_NOT_READY;
    }
  cudaError_t e = dispatch_diag(c, c->pc_raw, stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_precond_setup: diagonal");
  const long long nb = (c->N + 255) / 256;
  precond_invert_kernel<<<dim3((unsigned)nb), 256, 0, stream>>>(c->N, c->ld, c->G, c->pc_raw, c->pc_inv64,
                                                                c->pc_inv32);
  count_launches(1);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return cuda_fail(e, "sint_precond_setup: invert");
  c->has_ch = false;
  if (c->pc_kind == 1)
    {
      if (int rc = ch_sgs_setup(c, stream))
        return rc;
      c->has_ch = true;
    }
  c->has_pc = true;
  return SINT_OK;
}

int sint_set_preconditioner_type(sint_ctx *c, int type)
{
  if (int e = check_ctx(c))
    return e;
  if (type != 0 && type != 1)
    {
      set_error("sint_set_preconditioner_type: type must be 0 (block-Jacobi) or 1 (Cahn-Hilliard Gauss-Seidel)");
      return SINT_ERR_ARG;
    }
  if (type != c->pc_kind)
    c->has_pc = false; // takes effect at the next set-up
  c->pc_kind = type;
  return SINT_OK;
}

int sint_ch_matrix_f64(sint_ctx *c, double *A, sint_stream_t stream)
{
  if (int e = check_ctx(c))
    return e;
  if (!c->has_ch)
    {
      set_error("sint_ch_matrix_f64: the Cahn-Hilliard matrix is not set up (preconditioner type 1 and "
                "sint_precond_setup first)");
      return SINT_ERR_NOT_READY;
    }
  if (int e = check_vec(A, "A"))
    return e;
  const size_t nk = c->grid.dim == 3 ? 27 : 9;
  const cudaError_t e =
    cudaMemcpyAsync(A, c->ch_A64, sizeof(double) * nk * 4 * c->ld, cudaMemcpyDeviceToDevice, stream);
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_ch_matrix_f64");
}

int sint_precond_apply_f64(sint_ctx *c, double *z, const double *r, sint_stream_t stream)
{
  if (int e = check_ctx(c))
    return e;
  if (!c->has_pc)
    {
      set_error("sint_precond_apply_f64: preconditioner not set up");
      return SINT_ERR_NOT_READY;
    }
  if (int e = check_vec(z, "z"))
    return e;
  if (int e = check_vec(r, "r"))
    return e;
  const long long nb = (c->N + 255) / 256;
  precond_apply_kernel<double><<<dim3((unsigned)nb), 256, 0, stream>>>(c->N, c->ld, c->G, c->pc_inv64, r, z);
  count_launches(1);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && c->has_ch) // Cahn-Hilliard block by the Gauss-Seidel sweeps
    e = ch_sgs_apply<double>(c, r, z, stream);
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_precond_apply_f64");
}

int sint_precond_apply_f32(sint_ctx *c, float *z, const float *r, sint_stream_t stream)
{
  if (int e = check_ctx(c))
    return e;
  if (!c->has_pc)
    {
      set_error("sint_precond_apply_f32: preconditioner not set up");
      return SINT_ERR_NOT_READY;
    }
  if (int e = check_vec(z, "z"))
    return e;
  if (int e = check_vec(r, "r"))
    return e;
  const long long nb = (c->N + 255) / 256;
  precond_apply_kernel<float><<<dim3((unsigned)nb), 256, 0, stream>>>(c->N, c->ld, c->G, c->pc_inv32, r, z);
  count_launches(1);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && c->has_ch) // Cahn-Hilliard block by the Gauss-Seidel sweeps
    e = ch_sgs_apply<float>(c, r, z, stream);
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_precond_apply_f32");
}

int sint_ac_inverse_diagonal_f64(sint_ctx *c, double *inv_diag, sint_stream_t stream)
{
  if (int e = check_ctx(c))
    return e;
  if (!c->has_pc)
    {
      set_error("sint_ac_inverse_diagonal_f64: preconditioner not set up");
      return SINT_ERR_NOT_READY;
    }
  if (int e = check_vec(inv_diag, "inv_diag"))
    return e;
  const cudaError_t e = cudaMemcpyAsync(inv_diag, c->pc_inv64 + 4 * c->ld, sizeof(double) * c->G * c->ld,
                                        cudaMemcpyDeviceToDevice, stream);
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_ac_inverse_diagonal_f64");
}

int sint_ch_blocks_f64(sint_ctx *c, double *blocks, sint_stream_t stream)
{
  if (int e = check_ctx(c))
    return e;
  if (!c->has_pc)
    {
      set_error("sint_ch_blocks_f64: preconditioner not set up");
      return SINT_ERR_NOT_READY;
    }
  if (int e = check_vec(blocks, "blocks"))
    return e;
  const cudaError_t e =
    cudaMemcpyAsync(blocks, c->pc_raw, sizeof(double) * 4 * c->ld, cudaMemcpyDeviceToDevice, stream);
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_ch_blocks_f64");
}

} // extern "C"
