// Damped Newton with restarted GMRES and the block preconditioner, all
// vectors resident on the device.
//
//   DampedNewtonSolver::solve      include/pf-applications/lac/solvers_nonlinear.h:247-357
//   NewtonSolverSolverControl      solvers_nonlinear.h:37-156 (convergence test)
//   TimeMarchingImplicit lambdas   time_integration/time_marching.h:129-241
//   SolverGMRESWrapper             lac/solvers_linear.h:57-117 -> deal.II SolverGMRES
//                                  (left preconditioning, classical Gram-Schmidt,
//                                  ReductionControl(l_max_iter, l_abs_tol, l_rel_tol))
//
// Mixed precision (inner_precision == 32): the Newton residual, update and
// norms stay FP64; GMRES runs on FP32 Krylov vectors with the FP32
// Jacobian-vector product and FP32 preconditioner, its Gram-Schmidt dot
// products and norms accumulate in FP64 and its Hessenberg matrix is FP64.
#include <cmath>
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
        (e = cudaMallocHost(&w->h_s, sizeof(double) * (MAX_MULTIDOT + 2))) != cudaSuccess)
      {
        const int rc = cuda_fail(e, "newton workspace allocation");
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

  // Restarted, left-preconditioned GMRES for J x = b with x0 = 0; classical
  // Gram-Schmidt with a second pass when the first one loses more than 30%
  // of the norm.  Returns SINT_OK / SINT_ERR_NO_CONVERGENCE; *its = iterations.
  template <typename R>
  static int gmres(Ctx *c, const sint_newton_params &prm, cudaStream_t s, int *its_out)
  {
    Workspace      *ws = c->ws;
    const long long n  = ws->nvec;
    const int       m  = ws->restart;
    R              *V = static_cast<R *>(ws->V), *w = static_cast<R *>(ws->w), *t = static_cast<R *>(ws->t);
    R              *b = static_cast<R *>(ws->b), *x = static_cast<R *>(ws->x);
    std::vector<double> H((m + 1) * m, 0.0), cs(m, 0.0), sn(m, 0.0), gv(m + 1, 0.0), y(m, 0.0);
    int    its = 0, rc;
    double tol = 0.0;
    bool   first = true;
    if ((rc = axpby<R>(n, 0.0, b, 0.0, x, s)))
      return rc;
    for (;;)
      {
        // w = P^-1 (b - J x)
        if (first)
          {
            if ((rc = prec<R>(c, w, b, s)))
              return rc;
          }
        else
          {
            if ((rc = jvp<R>(c, t, x, s)) || (rc = axpby<R>(n, 1.0, b, -1.0, t, s)) || (rc = prec<R>(c, w, t, s)))
              return rc;
          }
        if ((rc = multidot<R>(c, n, w, w, 0, 1, ws->d_s, s)) || (rc = fetch(ws, 1, s)))
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
        if ((rc = axpby<R>(n, 1.0 / beta, w, 0.0, V, s)))
          return rc;
        std::fill(gv.begin(), gv.end(), 0.0);
        gv[0]     = beta;
        int    k  = 0; // number of basis vectors beyond V_0 built in this cycle
        double res = beta;
        for (int j = 0; j < m; ++j)
          {
            ++its;
            R *vj = V + (long long)j * n;
            if ((rc = jvp<R>(c, t, vj, s)) || (rc = prec<R>(c, w, t, s)))
              return rc;
            // classical Gram-Schmidt: h = V^T w, w -= V h
            double *hcol = &H[j * (m + 1)];
            if ((rc = multidot<R>(c, n, w, V, n, j + 1, ws->d_s, s)) ||
                (rc = multiaxpy_norm2<R>(c, n, w, V, n, j + 1, ws->d_s, ws->d_s + MAX_MULTIDOT, s)))
              return rc;
            {
              cudaError_t e = cudaMemcpyAsync(ws->h_s, ws->d_s, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, s);
              if (e == cudaSuccess)
                e = cudaMemcpyAsync(ws->h_s + MAX_MULTIDOT, ws->d_s + MAX_MULTIDOT, sizeof(double),
                                    cudaMemcpyDeviceToHost, s);
              if (e == cudaSuccess)
                e = cudaStreamSynchronize(s);
              if (e != cudaSuccess)
                return cuda_fail(e, "GMRES: fetch Hessenberg column");
            }
            double hh = 0.0;
            for (int i = 0; i <= j; ++i)
              {
                hcol[i] = ws->h_s[i];
                hh += hcol[i] * hcol[i];
              }
            double nw2 = ws->h_s[MAX_MULTIDOT];
            if (nw2 < 0.49 * (hh + nw2))
              {
                // second Gram-Schmidt pass (norm dropped by more than 30%)
                if ((rc = multidot<R>(c, n, w, V, n, j + 1, ws->d_s, s)) ||
                    (rc = multiaxpy_norm2<R>(c, n, w, V, n, j + 1, ws->d_s, ws->d_s + MAX_MULTIDOT, s)))
                  return rc;
                cudaError_t e =
                  cudaMemcpyAsync(ws->h_s, ws->d_s, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess)
                  e = cudaMemcpyAsync(ws->h_s + MAX_MULTIDOT, ws->d_s + MAX_MULTIDOT, sizeof(double),
                                      cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess)
                  e = cudaStreamSynchronize(s);
                if (e != cudaSuccess)
                  return cuda_fail(e, "GMRES: fetch second pass");
                for (int i = 0; i <= j; ++i)
                  hcol[i] += ws->h_s[i];
                nw2 = ws->h_s[MAX_MULTIDOT];
              }
            const double nw = std::sqrt(std::max(nw2, 0.0));
            hcol[j + 1]     = nw;
            // apply the previous Givens rotations, then a new one
            for (int i = 0; i < j; ++i)
              {
                const double a = hcol[i], bb = hcol[i + 1];
                hcol[i]         = cs[i] * a + sn[i] * bb;
                hcol[i + 1]     = -sn[i] * a + cs[i] * bb;
              }
            const double a = hcol[j], bb = hcol[j + 1];
            const double rr = std::hypot(a, bb);
            cs[j]           = rr == 0.0 ? 1.0 : a / rr;
            sn[j]           = rr == 0.0 ? 0.0 : bb / rr;
            hcol[j]         = rr;
            hcol[j + 1]     = 0.0;
            gv[j + 1]       = -sn[j] * gv[j];
            gv[j]           = cs[j] * gv[j];
            res             = std::fabs(gv[j + 1]);
            k               = j + 1;
            if (!std::isfinite(res) || !std::isfinite(nw))
              {
                set_error("GMRES: non-finite Hessenberg entry");
                *its_out = its;
                return SINT_ERR_NO_CONVERGENCE;
              }
            if (nw == 0.0 || res <= tol || its >= prm.l_max_iter || j == m - 1)
              break;
            if ((rc = axpby<R>(n, 1.0 / nw, w, 0.0, V + (long long)(j + 1) * n, s)))
              return rc;
          }
        // back substitution H(0:k,0:k) y = g, then x += V y
        for (int i = k - 1; i >= 0; --i)
          {
            double sum = gv[i];
            for (int l = i + 1; l < k; ++l)
              sum -= H[l * (m + 1) + i] * y[l];
            y[i] = sum / H[i * (m + 1) + i];
          }
        {
          cudaError_t e = cudaMemcpyAsync(ws->d_y, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s);
          if (e != cudaSuccess)
            return cuda_fail(e, "GMRES: upload y");
          if ((rc = lincomb<R>(n, x, V, n, k, ws->d_y, s)))
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
  const cudaError_t e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_newton_solve");
}

} // extern "C"
