// Damped Newton with restarted GMRES and the block preconditioner, all
// vectors resident on the device.
//
//   DampedNewtonSolver::solve      include/pf-applications/lac/solvers_nonlinear.h:247-357
//   NewtonSolverSolverControl      solvers_nonlinear.h:37-156 (convergence test)
//   TimeMarchingImplicit lambdas   time_integration/time_marching.h:129-241
//   SolverGMRESWrapper             lac/solvers_linear.h:57-117 -> deal.II SolverGMRES
//                                  (left preconditioning -- right as an option --, classical Gram-Schmidt,
//                                  ReductionControl(l_max_iter, l_abs_tol, l_rel_tol))
//
// Mixed precision (inner_precision == 32): the Newton residual, update and
// norms stay FP64; GMRES runs on FP32 Krylov vectors with the FP32
// Jacobian-vector product and FP32 preconditioner, its Gram-Schmidt dot
// products and norms accumulate in FP64 and its Hessenberg matrix is FP64.
#include <cmath>
#include <limits>
#include <cstring>
#include <string>
#include <vector>

#include "sint_internal.h"
#include "sint_launch.h"

namespace sint
{
  struct Workspace
  {
    long long nvec      = 0; // C * ld
    int       restart   = 0;
    int       precision = 0;
    double   *r = nullptr, *du = nullptr, *tmp = nullptr; // FP64 Newton vectors
    void     *V = nullptr, *w = nullptr, *t = nullptr, *b = nullptr, *x = nullptr;
    double   *d_s = nullptr; // device scalars: [0, MAX_MULTIDOT) dots, [MAX_MULTIDOT] norm
    double   *h_s = nullptr; // pinned host mirror
    double   *d_y = nullptr; // device copy of the GMRES coefficients
    // device-resident Arnoldi state: Hessenberg matrix (column j at j * (restart + 1)),
    // Givens rotations, rotated right-hand side g, scalars {|w|, tol}, the re-orthogonalisation flag
    double  *d_H = nullptr, *d_cs = nullptr, *d_sn = nullptr, *d_g = nullptr, *d_sc = nullptr;
    int     *d_flag = nullptr;
    double2 *d_out = nullptr, *h_out = nullptr; // per iteration {|g_{j+1}|, status}
    double  *h_H   = nullptr;                   // pinned host copy of H and g at the end of a cycle
    cudaEvent_t ev[MAX_MULTIDOT] = {};
    // The Krylov loop runs on a private non-blocking stream (joined to the
    // caller's stream by two events) so that Arnoldi iteration j can be
    // captured once as a CUDA graph and replayed; a graph is updated in place
    // when a kernel argument it holds (the operator's physics: time weights,
    // mobility) or the kernel set (grain cut-off on or off) has changed since
    // its capture.
    cudaStream_t ps       = nullptr;
    cudaEvent_t  join_in  = nullptr, join_out = nullptr;
    struct IterGraph
    {
      cudaGraphExec_t exec  = nullptr;
      Phys            key   = {};
      const uint16_t *mask  = nullptr; // cell masks the captured kernels read (nullptr: no cut-off)
      AdvData         adv   = {};      // advection tables the captured kernels read (none: null pointers)
      int             periodic = 0;    // periodic directions of the captured kernels
      int             variant  = 0;    // bit 0: right preconditioning, bit 1: Gauss-Seidel CH block
      int             nodes = 0;
    } graphs[MAX_MULTIDOT];
    // [FP32 Krylov vectors][grain cut-off][advection][variant]: one eager
    // solve with this kernel set has run (lazy kernel set-up is done outside
    // any capture)
    bool warm[2][2][2][4] = {};
  };

  int free_workspace(Ctx *c)
  {
    if (!c->ws)
      return SINT_OK;
    Workspace *w = c->ws;
    cudaFree(w->r);
    cudaFree(w->du);
    cudaFree(w->tmp);
    cudaFree(w->V);
    cudaFree(w->w);
    cudaFree(w->t);
    cudaFree(w->b);
    cudaFree(w->x);
    cudaFree(w->d_s);
    cudaFree(w->d_y);
    cudaFreeHost(w->h_s);
    cudaFree(w->d_H);
    cudaFree(w->d_cs);
    cudaFree(w->d_sn);
    cudaFree(w->d_g);
    cudaFree(w->d_sc);
    cudaFree(w->d_flag);
    cudaFree(w->d_out);
    cudaFreeHost(w->h_out);
    cudaFreeHost(w->h_H);
    for (cudaEvent_t &e : w->ev)
      if (e)
        cudaEventDestroy(e);
    for (auto &g : w->graphs)
      if (g.exec)
        cudaGraphExecDestroy(g.exec);
    if (w->join_in)
      cudaEventDestroy(w->join_in);
    if (w->join_out)
      cudaEventDestroy(w->join_out);
    if (w->ps)
      cudaStreamDestroy(w->ps);
    delete w;
    c->ws = nullptr;
    return SINT_OK;
  }

  static int ensure_workspace(Ctx *c, int restart, int precision)
  {
    if (c->ws && c->ws->restart == restart && c->ws->precision == precision)
      return SINT_OK;
    free_workspace(c);
    Workspace *w = new Workspace();
    c->ws        = w;
    w->nvec      = (long long)c->C * c->ld;
    w->restart   = restart;
    w->precision = precision;
    const size_t rb  = precision == 32 ? sizeof(float) : sizeof(double);
    const size_t n64 = size_t(w->nvec) * sizeof(double);
    const size_t nr  = size_t(w->nvec) * rb;
    cudaError_t  e;
    if ((e = cudaMalloc(&w->r, n64)) != cudaSuccess || (e = cudaMalloc(&w->du, n64)) != cudaSuccess ||
        (e = cudaMalloc(&w->tmp, n64)) != cudaSuccess || (e = cudaMalloc(&w->V, nr * (restart + 1))) != cudaSuccess ||
        (e = cudaMalloc(&w->w, nr)) != cudaSuccess || (e = cudaMalloc(&w->t, nr)) != cudaSuccess ||
        (e = cudaMalloc(&w->b, nr)) != cudaSuccess || (e = cudaMalloc(&w->x, nr)) != cudaSuccess ||
        (e = cudaMalloc(&w->d_s, sizeof(double) * (MAX_MULTIDOT + 2))) != cudaSuccess ||
        (e = cudaMalloc(&w->d_y, sizeof(double) * (MAX_MULTIDOT + 2))) != cudaSuccess ||
        (e = cudaMallocHost(&w->h_s, sizeof(double) * (MAX_MULTIDOT + 2))) != cudaSuccess ||
        (e = cudaMalloc(&w->d_H, sizeof(double) * (restart + 1) * (restart + 1))) != cudaSuccess ||
        (e = cudaMalloc(&w->d_cs, sizeof(double) * (restart + 1))) != cudaSuccess ||
        (e = cudaMalloc(&w->d_sn, sizeof(double) * (restart + 1))) != cudaSuccess ||
        (e = cudaMalloc(&w->d_g, sizeof(double) * (restart + 2))) != cudaSuccess ||
        (e = cudaMalloc(&w->d_sc, sizeof(double) * 4)) != cudaSuccess ||
        (e = cudaMalloc(&w->d_flag, sizeof(int) * 4)) != cudaSuccess ||
        (e = cudaMalloc(&w->d_out, sizeof(double2) * (restart + 1))) != cudaSuccess ||
        (e = cudaMallocHost(&w->h_out, sizeof(double2) * (restart + 1))) != cudaSuccess ||
        (e = cudaMallocHost(&w->h_H, sizeof(double) * ((restart + 1) * (restart + 1) + restart + 2))) != cudaSuccess)
      {
        const int rc = cuda_fail(e, "newton workspace allocation");
        free_workspace(c);
        return rc;
      }
    for (int j = 0; j <= restart; ++j)
      if ((e = cudaEventCreateWithFlags(&w->ev[j], cudaEventDisableTiming)) != cudaSuccess)
        {
          const int rc = cuda_fail(e, "newton workspace events");
          free_workspace(c);
          return rc;
        }
    if ((e = cudaStreamCreateWithFlags(&w->ps, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&w->join_in, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&w->join_out, cudaEventDisableTiming)) != cudaSuccess)
      {
        const int rc = cuda_fail(e, "newton workspace stream");
        free_workspace(c);
        return rc;
      }
    // padding entries take part in dot products: keep every vector zeroed
    if ((e = cudaMemset(w->r, 0, n64)) != cudaSuccess || (e = cudaMemset(w->du, 0, n64)) != cudaSuccess ||
        (e = cudaMemset(w->tmp, 0, n64)) != cudaSuccess || (e = cudaMemset(w->V, 0, nr * (restart + 1))) != cudaSuccess ||
        (e = cudaMemset(w->w, 0, nr)) != cudaSuccess || (e = cudaMemset(w->t, 0, nr)) != cudaSuccess ||
        (e = cudaMemset(w->b, 0, nr)) != cudaSuccess || (e = cudaMemset(w->x, 0, nr)) != cudaSuccess)
      {
        const int rc = cuda_fail(e, "newton workspace memset");
        free_workspace(c);
        return rc;
      }
    return SINT_OK;
  }

  // read `m` device doubles from ws->d_s to the host (synchronises the stream)
  static int fetch(Workspace *w, int m, cudaStream_t s)
  {
    cudaError_t e = cudaMemcpyAsync(w->h_s, w->d_s, sizeof(double) * m, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "fetch scalars");
  }

  template <typename R>
  static int jvp(Ctx *c, R *dst, const R *src, cudaStream_t s);
  template <>
  int jvp<double>(Ctx *c, double *dst, const double *src, cudaStream_t s)
  {
    return sint_jvp_f64(static_cast<sint_ctx *>(c), dst, src, s);
  }
  template <>
  int jvp<float>(Ctx *c, float *dst, const float *src, cudaStream_t s)
  {
    return sint_jvp_f32(static_cast<sint_ctx *>(c), dst, src, s);
  }
  template <typename R>
  static int prec(Ctx *c, R *z, const R *r, cudaStream_t s);
  template <>
  int prec<double>(Ctx *c, double *z, const double *r, cudaStream_t s)
  {
    return sint_precond_apply_f64(static_cast<sint_ctx *>(c), z, r, s);
  }
  template <>
  int prec<float>(Ctx *c, float *z, const float *r, cudaStream_t s)
  {
    return sint_precond_apply_f32(static_cast<sint_ctx *>(c), z, r, s);
  }

  // --- device-resident Arnoldi bookkeeping ------------------------------------
  // One thread does the O(restart) scalar work of an Arnoldi step on the GPU,
  // so the host never waits for a Hessenberg column: it only reads the
  // residual estimate of iteration j while iteration j + 1 already runs.

  // start of a cycle: g = (beta, 0, ...), sc[1] = tol (first cycle) and status
  __global__ void gmres_cycle_init_kernel(int m, double beta, double *g)
  {
    for (int i = threadIdx.x; i <= m; i += blockDim.x)
      g[i] = i == 0 ? beta : 0.0;
  }

  // after the first Gram-Schmidt pass: Hessenberg column j = h and deal.II's
  // re-orthogonalisation test (Kelley 1995, as in SolverGMRES): once |w| after
  // the pass falls below 10 sqrt(eps) of |w| before it, every later iteration
  // of this solve takes a second pass (the flag is sticky).  thresh2 =
  // 100 eps of the Krylov vectors' precision; |w|^2 before = |h|^2 + |w'|^2.
  __global__ void arnoldi_check_kernel(int j, int ldh, const double *__restrict__ d_s, double *__restrict__ H,
                                       double thresh2, int *__restrict__ reorth)
  {
    if (threadIdx.x != 0)
      return;
    double *hcol = H + (long long)j * ldh;
    double  hh   = 0.0;
    for (int i = 0; i <= j; ++i)
      {
        hcol[i] = d_s[i];
        hh += d_s[i] * d_s[i];
      }
    const double nw2 = d_s[MAX_MULTIDOT];
    if (nw2 < thresh2 * (hh + nw2))
      *reorth = 1;
  }

  // after the (optional) second pass: |w|, Givens rotations, residual estimate.
  // out[j] = {|g_{j+1}|, status}: 0 continue, 1 converged, 2 breakdown, 3 non-finite
  __global__ void arnoldi_finish_kernel(int j, int ldh, const double *__restrict__ d_s, double *__restrict__ H,
                                        double *__restrict__ cs, double *__restrict__ sn, double *__restrict__ g,
                                        const int *__restrict__ reorth, double *__restrict__ sc,
                                        double2 *__restrict__ out)
  {
    if (threadIdx.x != 0)
      return;
    double *hcol = H + (long long)j * ldh;
    if (*reorth)
      for (int i = 0; i <= j; ++i)
        hcol[i] += d_s[i];
    const double nw = sqrt(fmax(d_s[MAX_MULTIDOT], 0.0));
    hcol[j + 1]     = nw;
    for (int i = 0; i < j; ++i)
      {
        const double a = hcol[i], b = hcol[i + 1];
        hcol[i]         = cs[i] * a + sn[i] * b;
        hcol[i + 1]     = -sn[i] * a + cs[i] * b;
      }
    const double a = hcol[j], b = hcol[j + 1];
    const double rr = hypot(a, b);
    cs[j]           = rr == 0.0 ? 1.0 : a / rr;
    sn[j]           = rr == 0.0 ? 0.0 : b / rr;
    hcol[j]         = rr;
    hcol[j + 1]     = 0.0;
    g[j + 1]        = -sn[j] * g[j];
    g[j]            = cs[j] * g[j];
    const double res = fabs(g[j + 1]);
    double       status;
    if (!isfinite(res) || !isfinite(nw))
      status = 3.0;
    else if (res <= sc[1])
      status = 1.0;
    else if (nw == 0.0)
      status = 2.0;
    else
      status = 0.0;
    sc[0]  = nw;
    out[j] = make_double2(res, status);
  }

  // Restarted, left-preconditioned GMRES for J x = b with x0 = 0; classical
  // Gram-Schmidt with deal.II's re-orthogonalisation test (second pass from
  // the first iteration whose norm drops below 10 sqrt(eps) of its starting
  // value on).  Returns SINT_OK / SINT_ERR_NO_CONVERGENCE; *its = iterations.
  //
  // Each Arnoldi iteration is a fixed sequence of kernels (J v, P^-1, fused
  // multi-dot, fused multi-axpy + norm, check, conditional second pass,
  // finish, normalisation of the next basis vector) plus a 16-byte copy of
  // its residual estimate; the host enqueues iteration j + 1 before it waits
  // for iteration j's estimate, unless the residual history predicts that j
  // converges.  An iteration enqueued past convergence only writes basis
  // vector j + 2 and Hessenberg column j + 1, which the solution update
  // (columns 0..j) never reads.
  // Kernel-sequence variant of an Arnoldi iteration: bit 0 = right
  // preconditioning, bit 1 = the Gauss-Seidel Cahn-Hilliard block.
  static int gmres_variant(const Ctx *c, const sint_newton_params &prm)
  {
    return (prm.right_preconditioning ? 1 : 0) | (c->has_ch ? 2 : 0);
  }

  template <typename R>
  static int gmres_body(Ctx *c, const sint_newton_params &prm, cudaStream_t s, int *its_out)
  {
    Workspace      *ws = c->ws;
    const long long n  = ws->nvec;
    const int       m  = ws->restart, ldh = m + 1;
    R              *V = static_cast<R *>(ws->V), *w = static_cast<R *>(ws->w), *t = static_cast<R *>(ws->t);
    R              *b = static_cast<R *>(ws->b), *x = static_cast<R *>(ws->x);
    // grain cut-off: every GMRES vector is zero on the DoFs no relevant cell
    // touches (no residual, Jacobian or preconditioner entry reaches them),
    // so the BLAS steps skip those chunks; results are bitwise the same
    const uint32_t *live = active_live(c);
    std::vector<double> y(m, 0.0);
    int    its = 0, rc;
    double tol = 0.0;
    bool   first = true;
    // 100 eps of the Krylov vectors' precision: (10 sqrt(eps))^2
    const double reorth_thresh2 = 100.0 * double(std::numeric_limits<R>::epsilon());
    {
      // re-orthogonalisation starts off for every solve (deal.II: force_re_orthogonalization = false)
      const cudaError_t e = cudaMemsetAsync(ws->d_flag, 0, sizeof(int), s);
      if (e != cudaSuccess)
        return cuda_fail(e, "GMRES: reset");
    }

    const bool right   = prm.right_preconditioning != 0;
    const int  variant = gmres_variant(c, prm);
    auto enqueue_kernels = [&](int j) -> int {
      R  *vj = V + (long long)j * n;
      int r;
      // left: w = P^-1 J v_j; right: w = J P^-1 v_j
      if ((right ? ((r = prec<R>(c, t, vj, s)) || (r = jvp<R>(c, w, t, s)))
                 : ((r = jvp<R>(c, t, vj, s)) || (r = prec<R>(c, w, t, s)))) ||
          (r = multidot<R>(c, n, w, V, n, j + 1, ws->d_s, s, live)) ||
          (r = multiaxpy_norm2<R>(c, n, w, V, n, j + 1, ws->d_s, ws->d_s + MAX_MULTIDOT, s, live)))
        return r;
      arnoldi_check_kernel<<<1, 32, 0, s>>>(j, ldh, ws->d_s, ws->d_H, reorth_thresh2, ws->d_flag);
      count_launches(1);
      if ((r = multidot_if<R>(c, n, w, V, n, j + 1, ws->d_s, ws->d_flag, s, live)) ||
          (r = multiaxpy_norm2_if<R>(c, n, w, V, n, j + 1, ws->d_s, ws->d_s + MAX_MULTIDOT, ws->d_flag, s, live)))
        return r;
      arnoldi_finish_kernel<<<1, 32, 0, s>>>(j, ldh, ws->d_s, ws->d_H, ws->d_cs, ws->d_sn, ws->d_g, ws->d_flag,
                                             ws->d_sc, ws->d_out);
      count_launches(1);
      if ((r = scale_by_device<R>(n, w, ws->d_sc, V + (long long)(j + 1) * n, s, live)))
        return r;
      const cudaError_t e =
        cudaMemcpyAsync(ws->h_out + j, ws->d_out + j, sizeof(double2), cudaMemcpyDeviceToHost, s);
      return e == cudaSuccess ? SINT_OK : cuda_fail(e, "GMRES: enqueue");
    };

    // Iteration j: replay its graph (capture or update it first when needed),
    // then record the event the host waits on.
    auto enqueue = [&](int j) -> int {
      int r = SINT_OK;
      const AdvData adv = c->adv ? c->adv_view : AdvData();
      if (!ws->warm[sizeof(R) == 4][c->cut][c->adv][variant])
        r = enqueue_kernels(j);
      else
        {
          auto &g = ws->graphs[j];
          if (!g.exec || std::memcmp(&g.key, &c->phys, sizeof(Phys)) != 0 || g.mask != active_mask(c) ||
              std::memcmp(&g.adv, &adv, sizeof(AdvData)) != 0 || g.periodic != c->grid.periodic ||
              g.variant != variant)
            {
              cudaGraph_t       graph = nullptr;
              const long long   n0    = sint_kernel_launch_count();
              cudaError_t       e     = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
              if (e != cudaSuccess)
                return cuda_fail(e, "GMRES: begin capture");
              const int rk = enqueue_kernels(j);
              e            = cudaStreamEndCapture(s, &graph);
              count_launches(-int(sint_kernel_launch_count() - n0)); // captured, not launched
              if (rk != SINT_OK || e != cudaSuccess)
                {
                  if (graph)
                    cudaGraphDestroy(graph);
                  return rk != SINT_OK ? rk : cuda_fail(e, "GMRES: end capture");
                }
              size_t nn = 0;
              cudaGraphGetNodes(graph, nullptr, &nn);
              bool updated = false;
              if (g.exec)
                {
                  cudaGraphExecUpdateResultInfo info;
                  updated = cudaGraphExecUpdate(g.exec, graph, &info) == cudaSuccess;
                  if (!updated)
                    {
                      cudaGetLastError(); // clear the update failure; instantiate anew
                      cudaGraphExecDestroy(g.exec);
                      g.exec = nullptr;
                    }
                }
              if (!updated)
                e = cudaGraphInstantiate(&g.exec, graph, 0);
              cudaGraphDestroy(graph);
              if (e != cudaSuccess)
                {
                  g.exec = nullptr;
                  return cuda_fail(e, "GMRES: instantiate");
                }
              g.key   = c->phys;
              g.mask  = active_mask(c);
              g.adv   = adv;
              g.periodic = c->grid.periodic;
              g.variant  = variant;
              g.nodes = int(nn);
            }
          const cudaError_t e = cudaGraphLaunch(g.exec, s);
          if (e != cudaSuccess)
            return cuda_fail(e, "GMRES: graph launch");
          count_launches(g.nodes);
        }
      if (r != SINT_OK)
        return r;
      const cudaError_t e = cudaEventRecord(ws->ev[j], s);
      return e == cudaSuccess ? SINT_OK : cuda_fail(e, "GMRES: record");
    };

    if ((rc = axpby<R>(n, 0.0, b, 0.0, x, s, live)))
      return rc;
    for (;;)
      {
        // left: w = P^-1 (b - J x); right: w = b - J x
        if (first)
          {
            if ((rc = right ? axpby<R>(n, 1.0, b, 0.0, w, s, live) : prec<R>(c, w, b, s)))
              return rc;
          }
        else
          {
            if ((rc = jvp<R>(c, t, x, s)) || (rc = axpby<R>(n, 1.0, b, -1.0, t, s, live)) ||
                (rc = right ? axpby<R>(n, 1.0, t, 0.0, w, s, live) : prec<R>(c, w, t, s)))
              return rc;
          }
        if ((rc = multidot<R>(c, n, w, w, 0, 1, ws->d_s, s, live)) || (rc = fetch(ws, 1, s)))
          return rc;
        const double beta = std::sqrt(ws->h_s[0]);
        if (!std::isfinite(beta))
          {
            set_error("GMRES: non-finite residual");
            *its_out = its;
            return SINT_ERR_NO_CONVERGENCE;
          }
        if (first)
          {
            // deal.II ReductionControl: tolerance = max(abs_tol, rel_tol * |r0|)
            tol   = std::max(prm.l_abs_tol, prm.l_rel_tol * beta);
            first = false;
            const double sc[2] = {0.0, tol};
            cudaError_t  e     = cudaMemcpyAsync(ws->d_sc, sc, sizeof(sc), cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess)
              return cuda_fail(e, "GMRES: tolerance");
          }
        if (beta <= tol)
          {
            *its_out = its;
            return SINT_OK;
          }
        if (its >= prm.l_max_iter)
          {
            set_error("GMRES: maximum number of iterations reached");
            *its_out = its;
            return SINT_ERR_NO_CONVERGENCE;
          }
        if ((rc = axpby<R>(n, 1.0 / beta, w, 0.0, V, s, live)))
          return rc;
        gmres_cycle_init_kernel<<<1, 64, 0, s>>>(m, beta, ws->d_g);
        count_launches(1);

        int    k = 0, status = 0;
        double res = beta, res_prev = beta, res_prev2 = 0.0;
        bool   queued = false; // iteration j + 1 already enqueued
        if ((rc = enqueue(0)))
          return rc;
        for (int j = 0;; ++j)
          {
            queued = false;
            if (j + 1 < m && its + 1 < prm.l_max_iter)
              {
                // predicted estimate of iteration j from the last two (geometric decay)
                const double pred = res_prev2 > 0.0 ? res_prev * (res_prev / res_prev2) : 0.5 * res_prev;
                if (pred > tol)
                  {
                    if ((rc = enqueue(j + 1)))
                      return rc;
                    queued = true;
                  }
              }
            cudaError_t e = cudaEventSynchronize(ws->ev[j]);
            if (e != cudaSuccess)
              return cuda_fail(e, "GMRES: wait for iteration");
            ++its;
            k      = j + 1;
            res    = ws->h_out[j].x;
            status = int(ws->h_out[j].y);
            if (status == 3)
              {
                set_error("GMRES: non-finite Hessenberg entry");
                *its_out = its;
                return SINT_ERR_NO_CONVERGENCE;
              }
            if (status != 0 || its >= prm.l_max_iter || j == m - 1)
              break;
            if (!queued && (rc = enqueue(j + 1)))
              return rc;
            res_prev2 = res_prev;
            res_prev  = res;
          }
        // back substitution H(0:k,0:k) y = g on the host (k <= restart), then x += V y
        {
          cudaError_t e = cudaMemcpyAsync(ws->h_H, ws->d_H, sizeof(double) * ldh * k, cudaMemcpyDeviceToHost, s);
          if (e == cudaSuccess)
            e = cudaMemcpyAsync(ws->h_H + ldh * ldh, ws->d_g, sizeof(double) * k, cudaMemcpyDeviceToHost, s);
          if (e == cudaSuccess)
            e = cudaStreamSynchronize(s);
          if (e != cudaSuccess)
            return cuda_fail(e, "GMRES: fetch Hessenberg");
        }
        const double *H = ws->h_H, *gv = ws->h_H + ldh * ldh;
        for (int i = k - 1; i >= 0; --i)
          {
            double sum = gv[i];
            for (int l = i + 1; l < k; ++l)
              sum -= H[l * ldh + i] * y[l];
            y[i] = sum / H[i * ldh + i];
          }
        {
          cudaError_t e = cudaMemcpyAsync(ws->d_y, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s);
          if (e != cudaSuccess)
            return cuda_fail(e, "GMRES: upload y");
          if (right)
            {
              // x += P^-1 (V y)
              if ((rc = axpby<R>(n, 0.0, b, 0.0, t, s, live)) || (rc = lincomb<R>(n, t, V, n, k, ws->d_y, s, live)) ||
                  (rc = prec<R>(c, w, t, s)) || (rc = axpby<R>(n, 1.0, w, 1.0, x, s, live)))
                return rc;
            }
          else if ((rc = lincomb<R>(n, x, V, n, k, ws->d_y, s, live)))
            return rc;
          // y lives in a host vector that the next cycle overwrites
          if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
            return cuda_fail(e, "GMRES: sync");
        }
        if (res <= tol)
          {
            *its_out = its;
            return SINT_OK;
          }
        if (its >= prm.l_max_iter)
          {
            set_error("GMRES: maximum number of iterations reached");
            *its_out = its;
            return SINT_ERR_NO_CONVERGENCE;
          }
      }
  }

  // GMRES on the workspace's private stream, ordered after and before the caller's stream.
  template <typename R>
  static int gmres(Ctx *c, const sint_newton_params &prm, cudaStream_t s, int *its_out)
  {
    Workspace  *ws = c->ws;
    cudaError_t e  = cudaEventRecord(ws->join_in, s);
    if (e == cudaSuccess)
      e = cudaStreamWaitEvent(ws->ps, ws->join_in, 0);
    if (e != cudaSuccess)
      return cuda_fail(e, "GMRES: join");
    const int rc = gmres_body<R>(c, prm, ws->ps, its_out);
    e            = cudaEventRecord(ws->join_out, ws->ps);
    if (e == cudaSuccess)
      e = cudaStreamWaitEvent(s, ws->join_out, 0);
    if (e != cudaSuccess)
      return cuda_fail(e, "GMRES: join back");
    if (rc == SINT_OK)
      ws->warm[sizeof(R) == 4][c->cut][c->adv][gmres_variant(c, prm)] = true;
    return rc;
  }

  static int residual_norm(Ctx *c, double *r, double *out, cudaStream_t s)
  {
    Workspace *ws = c->ws;
    int        rc;
    if ((rc = dot_f64(c, ws->nvec, r, r, ws->d_s, s)) || (rc = fetch(ws, 1, s)))
      return rc;
    *out = std::sqrt(ws->h_s[0]);
    return SINT_OK;
  }
} // namespace sint

using namespace sint;

extern "C" {

void sint_newton_default_params(sint_newton_params *p)
{
  if (!p)
    return;
  p->nl_max_iter           = 10;
  p->nl_abs_tol            = 1e-20;
  p->nl_rel_tol            = 1e-5;
  p->l_max_iter            = 1000;
  p->l_abs_tol             = 1e-10;
  p->l_rel_tol             = 1e-2;
  p->gmres_restart         = 30;
  p->threshold_newton_iter = 100;
  p->threshold_linear_iter = 20;
  p->use_damping           = 1;
  p->reuse_preconditioner  = 1;
  p->inner_precision       = 64;
  p->right_preconditioning = 0;
}

int sint_newton_clear(sint_ctx *c)
{
  if (!c)
    {
      set_error("sint_newton_clear: null context");
      return SINT_ERR_ARG;
    }
  c->history_newton_iterations      = 0;
  c->history_linear_iterations_last = 0;
  return SINT_OK;
}

int sint_newton_solve(sint_ctx *c, double *u, const double *const *hist, const sint_newton_params *prm_in,
                      sint_newton_stats *stats, sint_stream_t s)
{
  if (!c || !u)
    {
      set_error("sint_newton_solve: null argument");
      return SINT_ERR_ARG;
    }
  sint_newton_params prm;
  if (prm_in)
    prm = *prm_in;
  else
    sint_newton_default_params(&prm);
  if (prm.gmres_restart < 1 || prm.gmres_restart > MAX_MULTIDOT - 1 ||
      (prm.inner_precision != 32 && prm.inner_precision != 64) || prm.nl_max_iter < 0 || prm.l_max_iter < 1 ||
      prm.threshold_newton_iter < 1)
    {
      set_error("sint_newton_solve: invalid parameters");
      return SINT_ERR_ARG;
    }
  if (c->phys.order < 1 || !hist)
    {
      set_error("sint_newton_solve: time weights of order >= 1 and the history are required");
      return SINT_ERR_ARG;
    }
  int rc;
  if ((rc = ensure_workspace(c, prm.gmres_restart, prm.inner_precision)))
    return rc;
  Workspace        *ws = c->ws;
  const long long   n  = ws->nvec;
  sint_newton_stats st;
  std::memset(&st, 0, sizeof(st));
  if (!prm.reuse_preconditioner)
    sint_newton_clear(c);

  // residual(u) -> r, |r|
  if ((rc = sint_residual_f64(c, ws->r, u, hist, 2, s)))
    return rc;
  st.residual_evaluations++;
  double norm_r;
  if ((rc = residual_norm(c, ws->r, &norm_r, s)))
    return rc;
  st.initial_residual = st.final_residual = norm_r;
  const double norm_0 = norm_r;

  // NewtonSolverSolverControl::check (solvers_nonlinear.h:92-117)
  auto check = [&](int step, double v) -> int {
    if (v > prm.nl_abs_tol && v / norm_0 > prm.nl_rel_tol && step < prm.nl_max_iter)
      return 0; // iterate
    if (v <= prm.nl_abs_tol || v / norm_0 <= prm.nl_rel_tol)
      return 1; // success
    return 2;   // failure
  };

  int status = check(0, norm_r);
  int it     = 0;
  while (status == 0)
    {
      // increment = 0, r *= -1
      if ((rc = axpby<double>(n, 0.0, ws->r, -1.0, ws->r, s)))
        return rc;
      const bool threshold_exceeded = (c->history_newton_iterations % prm.threshold_newton_iter == 0) ||
                                      ((int)c->history_linear_iterations_last > prm.threshold_linear_iter);
      // setup_jacobian (time_marching.h:139-165)
      if ((rc = sint_set_linearization_point(c, u, s)))
        return rc;
      st.jacobian_setups++;
      // setup_preconditioner (time_marching.h:168-207)
      if (threshold_exceeded || !c->has_pc)
        {
          if ((rc = sint_precond_setup(c, s)))
            return rc;
          st.preconditioner_setups++;
        }
      // solve_with_jacobian (time_marching.h:210-241)
      int lits = 0;
      if (prm.inner_precision == 32)
        {
          if ((rc = convert<double, float>(n, ws->r, static_cast<float *>(ws->b), s)))
            return rc;
          rc = gmres<float>(c, prm, s, &lits);
          if (rc == SINT_OK)
            rc = convert<float, double>(n, static_cast<float *>(ws->x), ws->du, s);
        }
      else
        {
          if ((rc = axpby<double>(n, 1.0, ws->r, 0.0, static_cast<double *>(ws->b), s)))
            return rc;
          rc = gmres<double>(c, prm, s, &lits);
          if (rc == SINT_OK)
            rc = axpby<double>(n, 1.0, static_cast<double *>(ws->x), 0.0, ws->du, s);
        }
      st.linear_iterations += lits;
      c->history_linear_iterations_last = lits;
      if (rc)
        {
          st.newton_iterations = it;
          st.final_residual    = norm_r;
          if (stats)
            *stats = st;
          return rc;
        }

      double norm_new = 0.0;
      if (prm.use_damping)
        {
          // damped Newton scheme (solvers_nonlinear.h:294-333)
          const double tau   = 0.1;
          double       omega = 1.0;
          int          n_tmp = 0;
          do
            {
              if ((rc = axpby<double>(n, 1.0, u, 0.0, ws->tmp, s)) ||
                  (rc = axpby<double>(n, omega, ws->du, 1.0, ws->tmp, s)) ||
                  (rc = sint_residual_f64(c, ws->r, ws->tmp, hist, 2, s)))
                return rc;
              st.residual_evaluations++;
              if ((rc = residual_norm(c, ws->r, &norm_new, s)))
                return rc;
              omega = omega / 2.0;
              n_tmp++;
          } while (norm_new >= (1.0 - tau * omega) * norm_r && n_tmp < 100);
          if (!(norm_new < (1.0 - tau * omega) * norm_r))
            {
              set_error("Maximum number of damping iterations of damp Netwon exceeded!");
              st.newton_iterations = it;
              st.final_residual    = norm_r;
              if (stats)
                *stats = st;
              return SINT_ERR_NEWTON;
            }
          if ((rc = axpby<double>(n, 1.0, ws->tmp, 0.0, u, s)))
            return rc;
        }
      else
        {
          if ((rc = axpby<double>(n, 1.0, ws->du, 1.0, u, s)) || (rc = sint_residual_f64(c, ws->r, u, hist, 2, s)))
            return rc;
          st.residual_evaluations++;
          if ((rc = residual_norm(c, ws->r, &norm_new, s)))
            return rc;
        }
      norm_r = norm_new;
      ++it;
      ++c->history_newton_iterations;
      status = check(it, norm_r);
    }
  st.newton_iterations = it;
  st.final_residual    = norm_r;
  if (stats)
    *stats = st;
  if (status != 1)
    {
      set_error(std::isfinite(norm_r) ? "Maximum number of Newton iterations of damp Netwon exceeded!"
                                      : "Newton: non-finite residual");
      return SINT_ERR_NEWTON;
    }
  // periodic constraints: the slave entries of the converged step follow
  // their masters (the updates leave them untouched: J v has identity rows
  // and the residual zero rows there)
  cudaError_t e = launch_periodic_distribute(c->grid, c->C, u, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_newton_solve");
}

} // extern "C"
