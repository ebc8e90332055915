// CPU oracle for the sintering operator: TEST INFRASTRUCTURE ONLY.
//
// A plain FP64 restatement of hpsint's generic Cahn-Hilliard/Allen-Cahn
// sintering operator on uniform Cartesian Q1 meshes (FE_Q(1), QGauss(2),
// affine cells), written for readability, not speed.  Only the test-suite,
// the package's smoke check and the CPU-baseline leg of the benchmark may
// load it; the CUDA product never links or calls it.
//
// Each function names the reference lines (paths inside the hpsint project)
// whose arithmetic it restates.  deal.II's MatrixFree/FEEvaluation is not
// available here, so its cell evaluation is restated from the finite-element
// definitions: tensor-product Q1 shape functions on [0,1]^dim, the 2-point
// Gauss rule (points 1/2 -+ 1/(2 sqrt 3), weights 1/2), JxW = prod(h_d / 2).
//
// Vector layout: C = G + 2 blocks (c, mu, eta_1..eta_G), block b holds the
// N nodal values of component b in lexicographic node order
// (x fastest, then y, then z), blocks are contiguous with stride N.
//
// Cell loops are parallelised with OpenMP over 2^dim cell colours (parity of
// the cell index in each direction); cells of one colour share no node, so
// the scatter is race-free and the summation order deterministic.
//
// Grain cut-off: with a cell mask (one uint16 per cell, bit b = grain b
// relevant, cells in lexicographic order) a cell gathers c, mu and its
// relevant grains only, runs the point physics with that many grains and
// scatters into those blocks only -- the src_view / vector_indices loops of
// do_vmult_range_no_template and do_evaluate_nonlinear_residual_nt
// (sintering/operator_sintering_generic.h:456-537, :1008-1081).  A null mask
// keeps every grain.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace
{
  constexpr int MAXG = 16;
  constexpr int MAXC = MAXG + 2;

  struct V3
  {
    double x[3] = {0.0, 0.0, 0.0};
    double &operator[](int i) { return x[i]; }
    double  operator[](int i) const { return x[i]; }
  };
  inline V3 operator+(const V3 &a, const V3 &b) { V3 r; for (int i = 0; i < 3; ++i) r[i] = a[i] + b[i]; return r; }
  inline V3 operator-(const V3 &a, const V3 &b) { V3 r; for (int i = 0; i < 3; ++i) r[i] = a[i] - b[i]; return r; }
  inline V3 operator*(const V3 &a, double s) { V3 r; for (int i = 0; i < 3; ++i) r[i] = a[i] * s; return r; }
  inline V3 operator*(double s, const V3 &a) { return a * s; }
  inline double dot(const V3 &a, const V3 &b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
  inline V3 &operator+=(V3 &a, const V3 &b) { for (int i = 0; i < 3; ++i) a[i] += b[i]; return a; }

  struct M3
  {
    double a[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  };
  inline V3 mul(const M3 &m, const V3 &v)
  {
    V3 r;
    for (int i = 0; i < 3; ++i)
      r[i] = m.a[i][0] * v[0] + m.a[i][1] * v[1] + m.a[i][2] * v[2];
    return r;
  }
  inline M3 mul(const M3 &m, const M3 &n)
  {
    M3 r;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        r.a[i][j] = m.a[i][0] * n.a[0][j] + m.a[i][1] * n.a[1][j] + m.a[i][2] * n.a[2][j];
    return r;
  }

  // include/pf-applications/base/tensor.h:125-135 (diagonal_matrix); only the
  // first `dim` diagonal entries are set, as for a deal.II Tensor<2,dim>.
  inline M3 diagonal_matrix(int dim, double fac)
  {
    M3 r;
    for (int d = 0; d < dim; ++d)
      r.a[d][d] = fac;
    return r;
  }
  inline M3 outer(const V3 &a, const V3 &b)
  {
    M3 r;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        r.a[i][j] = a[i] * b[j];
    return r;
  }
  inline M3 add(const M3 &a, const M3 &b)
  {
    M3 r;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        r.a[i][j] = a.a[i][j] + b.a[i][j];
    return r;
  }
  inline M3 scale(const M3 &a, double s)
  {
    M3 r;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        r.a[i][j] = a.a[i][j] * s;
    return r;
  }
  inline double norm(const V3 &v) { return std::sqrt(dot(v, v)); }

  // tensor.h:137-154 unit_vector(vec, zero_tol = 1e-10)
  inline V3 unit_vector(const V3 &v, double zero_tol = 1e-10)
  {
    const double nrm    = norm(v);
    const double filter = nrm > zero_tol ? 1.0 : 0.0;
    const double fn     = nrm < zero_tol ? 1.0 : nrm;
    V3 r;
    for (int i = 0; i < 3; ++i)
      r[i] = (v[i] / fn) * filter;
    return r;
  }

  // tensor.h:156-174 unit_vector_filter_2(vec, zero_tol = 1e-20)
  inline double unit_vector_filter_2(const V3 &v, double zero_tol = 1e-20)
  {
    const double n2     = dot(v, v);
    const double filter = n2 > zero_tol ? 1.0 : 0.0;
    const double fn     = n2 < zero_tol ? 1.0 : n2;
    return filter / fn;
  }

  // tensor.h:176-186 projector_matrix(vec, fac, diag) = (diag*I - vec (x) vec) * fac
  inline M3 projector_matrix(int dim, const V3 &v, double fac, double diag = 1.0)
  {
    M3 t = diagonal_matrix(dim, diag);
    M3 o = outer(v, v);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        t.a[i][j] = (t.a[i][j] - o.a[i][j]) * fac;
    return t;
  }

  // ------------------------------------------------------------------------
  // Bulk free energy: sintering/free_energy.h:37-176 (Evaluation),
  // numerics/power_helper.h:31-45 (power sums)
  struct FreeEnergyEval
  {
    double A, B, c, s2, s3;

    FreeEnergyEval(double A_, double B_, const double *state, int G)
      : A(A_), B(B_), c(state[0]), s2(0.0), s3(0.0)
    {
      for (int i = 0; i < G; ++i)
        {
          const double e = state[2 + i];
          s2 += e * e;
          s3 += e * e * e;
        }
    }
    // free_energy.h:111-122
    double f() const
    {
      return A * (c * c) * ((-c + 1.0) * (-c + 1.0)) +
             B * ((c * c) + (-6.0 * c + 6.0) * s2 - (-4.0 * c + 8.0) * s3 + 3.0 * (s2 * s2));
    }
    // free_energy.h:124-134
    double df_dc() const
    {
      return A * (c * c) * (2.0 * c - 2.0) + 2.0 * A * c * ((-c + 1.0) * (-c + 1.0)) +
             B * (2.0 * c - 6.0 * s2 + 4.0 * s3);
    }
    // free_energy.h:136-141
    double df_detai(double e) const
    {
      return e * (B * 12.0) * (e * (1.0 * c - 2.0) + (-c + 1.0) + s2);
    }
    // free_energy.h:143-148
    double d2f_dc2() const
    {
      return 2.0 * A * (c * c) + 4.0 * A * c * (2.0 * c - 2.0) + 2.0 * A * ((-c + 1.0) * (-c + 1.0)) + 2.0 * B;
    }
    // free_energy.h:150-154
    double d2f_dcdetai(double e) const { return (B * 12.0) * e * (e - 1.0); }
    // free_energy.h:156-161
    double d2f_detai2(double e) const
    {
      return B * (12.0 - 12.0 * c + 2.0 * e * (12.0 * c - 24.0) + 24.0 * (e * e) + 12.0 * s2);
    }
    // free_energy.h:163-168
    double d2f_detaidetaj(double ei, double ej) const { return 24.0 * B * ei * ej; }
  };

  // free_energy.h:233-252 apply_d2f_detaidetaj
  inline void apply_d2f_detaidetaj(double B, double L, const double *etas, int G,
                                   const double *value, double *value_result)
  {
    if (G <= 1)
      return;
    double temp = etas[0] * value[0];
    for (int ig = 1; ig < G; ++ig)
      temp += etas[ig] * value[ig];
    for (int ig = 0; ig < G; ++ig)
      value_result[ig] += (L * 24.0 * B) * etas[ig] * (temp - etas[ig] * value[ig]);
  }
}

// --------------------------------------------------------------------------
// C interface (structs mirror the ones the tests build with ctypes)
extern "C" {

typedef struct
{
  int    dim;
  int    n[3];
  double h[3];
} oracle_mesh;

typedef struct
{
  int    n_grains;
  double A, B, kappa_c, kappa_p;
  double Mvol, Mvap, Msurf, Mgb, L;
  int    tensorial;
} oracle_params;

// Advection (rigid-body motion) data: cell_segments[b * n_cells + cell] =
// segment of order parameter b the cell belongs to (-1: none); segments[9 s
// ..] = translational velocity (3), angular velocity (3; z only in 2D) and
// center (3) of segment s, so the velocity at x is v_t + w x (x - center)
// (AdvectionMechanism::calc_translation_velocity / calc_rotation_velocity,
// sintering/advection.h:330-352).  origin = lower corner of the mesh.
typedef struct
{
  const int    *cell_segments;
  const double *segments;
  int           n_segments;
  double        origin[3];
} oracle_advection;

typedef struct
{
  double w0;        // primary BDF weight  (time_integrator_data.h:150-154)
  double w_alg;     // algebraic weight of the mu row (time_integrator_data.h:158-163)
  int    order;     // number of old solutions used by the history term
  double w_hist[4]; // weights[1..order] of the BDF scheme (time_schemes.h:64-153)
} oracle_time;

} // extern "C"

namespace
{
  // ------------------------------------------------------------------------
  // Mobility: sintering/mobility.h
  struct Mobility
  {
    int    dim;
    double Mvol, Mvap, Msurf, Mgb, L;
    bool   tensorial;
    static constexpr double projector_scale = 1.001; // mobility.h:960

    static double phi_clamped(double c)
    {
      double phi = c * c * c * (10.0 - 15.0 * c + 6.0 * c * c);
      phi        = std::max(0.0, phi);
      phi        = std::min(1.0, phi);
      return phi;
    }

    // scalar: mobility.h:439-472, tensorial: mobility.h:756-804
    V3 apply_M(double c, const double *etas, int G, const V3 &c_grad, const V3 *etas_grad, const V3 &mu_grad) const
    {
      if (!tensorial)
        {
          double etaijSum = 0.0;
          for (int i = 0; i < G; ++i)
            for (int j = 0; j < i; ++j)
              etaijSum += etas[i] * etas[j];
          const double phi = phi_clamped(c);
          const double M   = Mvol * phi + Mvap * (1.0 - phi) + Msurf * 4.0 * c * c * (1.0 - c) * (1.0 - c) +
                           (2.0 * Mgb) * etaijSum;
          return M * mu_grad;
        }
      const double phi       = phi_clamped(c);
      const double f_vol_vap = Mvol * phi + Mvap * (1.0 - phi);
      const double fsurf     = Msurf * 4.0 * (c * c) * ((1. - c) * (1. - c));
      const V3     nc        = unit_vector(c_grad);
      V3           out       = (f_vol_vap + fsurf * projector_scale) * mu_grad - nc * (fsurf * dot(nc, mu_grad));
      if (G <= 1)
        return out;
      V3 out_gb;
      for (int i = 0; i < G; ++i)
        for (int j = 0; j < i; ++j)
          {
            const V3     d      = etas_grad[i] - etas_grad[j];
            const double filter = unit_vector_filter_2(d);
            out_gb += (mu_grad - d * (filter * dot(d, mu_grad))) * (etas[i] * etas[j]);
          }
      return out + out_gb * (2.0 * Mgb);
    }

    // scalar: mobility.h:476-534, tensorial: mobility.h:808-916
    V3 apply_M_derivative(const double *lin_value, const V3 *lin_gradient, int G, const double *value,
                          const V3 *gradient) const
    {
      const double  lin_c    = lin_value[0];
      const double *lin_etas = lin_value + 2;
      const V3     &lin_mu_g = lin_gradient[1];
      const double  c_value  = value[0];
      const double *etas_val = value + 2;
      const V3     &mu_g     = gradient[1];

      if (!tensorial)
        {
          double eta_sum = 0.0, eta_ij_sum = 0.0;
          for (int i = 0; i < G; ++i)
            {
              eta_sum += lin_etas[i];
              for (int j = 0; j < i; ++j)
                eta_ij_sum += lin_etas[i] * lin_etas[j];
            }
          const double phi = phi_clamped(lin_c);
          const double M   = Mvol * phi + Mvap * (1.0 - phi) +
                           Msurf * 4.0 * lin_c * lin_c * (1.0 - lin_c) * (1.0 - lin_c) + (2.0 * Mgb) * eta_ij_sum;
          const double dphidc = 30.0 * lin_c * lin_c * (1.0 - lin_c) * (1.0 - lin_c);
          const double dMdc =
            Mvol * dphidc - Mvap * dphidc + Msurf * 8.0 * lin_c * (1.0 - 3.0 * lin_c + 2.0 * lin_c * lin_c);
          double factor = 0.0;
          for (int i = 0; i < G; ++i)
            factor += (eta_sum - lin_etas[i]) * etas_val[i];
          return M * mu_g + (dMdc * c_value + (2.0 * Mgb) * factor) * lin_mu_g;
        }

      const V3 &lin_c_g    = lin_gradient[0];
      const V3 *lin_etas_g = lin_gradient + 2;
      const V3 &c_g        = gradient[0];

      V3       out, out_gb;
      const V3 nc = unit_vector(lin_c_g);
      {
        const double phi       = phi_clamped(lin_c);
        const double f_vol_vap = Mvol * phi + Mvap * (1.0 - phi);
        const double fsurf     = Msurf * 4.0 * (lin_c * lin_c) * ((1. - lin_c) * (1. - lin_c));
        out                    = (f_vol_vap + fsurf) * mu_g - nc * (fsurf * dot(nc, mu_g));
      }
      {
        const double c2_1minusc2 = 4.0 * lin_c * lin_c * (1. - lin_c) * (1. - lin_c);
        const double dphidc      = 30.0 * c2_1minusc2;
        const double f_vol_vap   = (Mvol - Mvap) * dphidc;
        const double fsurf       = Msurf * c2_1minusc2;
        double       dfsurf      = Msurf * 8.0 * lin_c * (1. - lin_c) * (1. - 2. * lin_c);
        if (fsurf < 1e-6)
          dfsurf = 0.0;
        out += ((f_vol_vap + dfsurf * projector_scale) * lin_mu_g - nc * (dfsurf * dot(nc, lin_mu_g))) * c_value;
      }
      {
        double fsurf = Msurf * 4.0 * (lin_c * lin_c) * ((1. - lin_c) * (1. - lin_c));
        double nrm   = norm(lin_c_g);
        if (fsurf < 1e-6)
          fsurf = 0.0;
        if (nrm < 1e-4)
          nrm = 1.0;
        const V3 temp = c_g - nc * dot(nc, c_g);
        out += (-fsurf / nrm) * (dot(nc, lin_mu_g) * temp + nc * dot(lin_mu_g, temp));
      }
      if (G <= 1)
        return out;
      for (int i = 0; i < G; ++i)
        for (int j = 0; j < i; ++j)
          {
            const V3     d      = lin_etas_g[i] - lin_etas_g[j];
            const double filter = unit_vector_filter_2(d);
            out_gb += (mu_g - d * (filter * dot(d, mu_g))) * (lin_etas[i] * lin_etas[j]);
            out_gb += (lin_mu_g - (d * filter) * dot(d, lin_mu_g)) *
                      (lin_etas[j] * etas_val[i] + lin_etas[i] * etas_val[j]);
          }
      return out + out_gb * (2.0 * Mgb);
    }

    // scalar: mobility.h:378-394 (returns the scalar times identity),
    // tensorial: mobility.h:668-696
    M3 dM_dc(double c, const V3 &c_grad) const
    {
      if (!tensorial)
        {
          const double dphidc = 30.0 * c * c * (1.0 - c) * (1.0 - c);
          const double dMdc   = Mvol * dphidc - Mvap * dphidc + Msurf * 8.0 * c * (1.0 - 3.0 * c + 2.0 * c * c);
          return diagonal_matrix(dim, dMdc);
        }
      const double c2_1minusc2 = 4.0 * c * c * (1. - c) * (1. - c);
      const double dphidc      = 30.0 * c2_1minusc2;
      M3           dMdc        = diagonal_matrix(dim, (Mvol - Mvap) * dphidc);
      const double fsurf       = Msurf * c2_1minusc2;
      double       dfsurf      = Msurf * 8.0 * c * (1. - c) * (1. - 2. * c);
      if (fsurf < 1e-6)
        dfsurf = 0.0;
      const V3 nc = unit_vector(c_grad);
      return add(dMdc, projector_matrix(dim, nc, dfsurf, projector_scale));
    }

    // scalar: mobility.h:399-409 (zero), tensorial: mobility.h:700-721
    M3 dM_dgrad_c(double c, const V3 &c_grad, const V3 &mu_grad) const
    {
      if (!tensorial)
        return M3();
      double fsurf = Msurf * 4.0 * (c * c) * ((1. - c) * (1. - c));
      double nrm   = norm(c_grad);
      if (fsurf < 1e-6)
        fsurf = 0.0;
      if (nrm < 1e-4)
        nrm = 1.0;
      const V3 nc = unit_vector(c_grad);
      const M3 M  = projector_matrix(dim, nc, 1. / nrm);
      M3       T  = add(diagonal_matrix(dim, dot(nc, mu_grad)), outer(nc, mu_grad));
      T           = scale(T, -fsurf);
      return mul(T, M);
    }
  };

  // ------------------------------------------------------------------------
  // Mesh / finite-element helpers
  struct Geometry
  {
    int     dim;
    int     n[3];  // cells per direction (n[2] = 1 in 2D)
    int     nn[3]; // nodes per direction (nn[2] = 1 in 2D)
    int64_t n_nodes;
    int64_t n_cells;
    double  h[3];
    int     nq;       // quadrature points = local nodes = 2^dim
    double  JxW;      // constant on the uniform affine mesh
    double  shape[8][8];     // shape[q][l]
    double  dshape[8][8][3]; // dshape[q][l][d]

    explicit Geometry(const oracle_mesh &m)
    {
      dim = m.dim;
      for (int d = 0; d < 3; ++d)
        {
          n[d]  = d < dim ? m.n[d] : 1;
          nn[d] = d < dim ? m.n[d] + 1 : 1;
          h[d]  = d < dim ? m.h[d] : 1.0;
        }
      n_nodes = int64_t(nn[0]) * nn[1] * nn[2];
      n_cells = int64_t(n[0]) * n[1] * n[2];
      nq      = 1 << dim;
      // 2-point Gauss-Legendre rule on [0,1]
      const double g[2] = {0.5 - 0.5 / std::sqrt(3.0), 0.5 + 0.5 / std::sqrt(3.0)};
      JxW               = 1.0;
      for (int d = 0; d < dim; ++d)
        JxW *= h[d] * 0.5;
      for (int q = 0; q < nq; ++q)
        for (int l = 0; l < nq; ++l)
          {
            double val = 1.0;
            double s1[3], ds1[3];
            for (int d = 0; d < dim; ++d)
              {
                const int    qd = (q >> d) & 1, ld = (l >> d) & 1;
                const double x  = g[qd];
                s1[d]           = ld ? x : 1.0 - x;
                ds1[d]          = (ld ? 1.0 : -1.0) / h[d];
                val *= s1[d];
              }
            shape[q][l] = val;
            for (int d = 0; d < 3; ++d)
              {
                double gr = 0.0;
                if (d < dim)
                  {
                    gr = ds1[d];
                    for (int e = 0; e < dim; ++e)
                      if (e != d)
                        gr *= s1[e];
                  }
                dshape[q][l][d] = gr;
              }
          }
    }

    // global index of local node l of cell (i,j,k)
    int64_t node(int i, int j, int k, int l) const
    {
      const int di = l & 1, dj = (l >> 1) & 1, dk = (l >> 2) & 1;
      return int64_t(i + di) + int64_t(nn[0]) * (int64_t(j + dj) + int64_t(nn[1]) * (k + dk));
    }
  };

  // Apply `body(i,j,k)` to every cell, colour by colour; within a colour the
  // cells are independent (no shared node) and run in parallel.
  template <typename Body>
  void coloured_cell_loop(const Geometry &geo, int n_threads, Body body)
  {
    const int n_colours = 1 << geo.dim;
    for (int colour = 0; colour < n_colours; ++colour)
      {
        const int ci = colour & 1, cj = (colour >> 1) & 1, ck = (colour >> 2) & 1;
        const int mi = (geo.n[0] - ci + 1) / 2, mj = (geo.n[1] - cj + 1) / 2,
                  mk = geo.dim == 3 ? (geo.n[2] - ck + 1) / 2 : 1;
        const int64_t total = int64_t(mi) * mj * mk;
#pragma omp parallel for schedule(static) num_threads(n_threads) if (n_threads > 1)
        for (int64_t t = 0; t < total; ++t)
          {
            const int a = int(t % mi), b = int((t / mi) % mj), c = int(t / (int64_t(mi) * mj));
            body(2 * a + ci, 2 * b + cj, geo.dim == 3 ? 2 * c + ck : 0);
          }
      }
  }

  // FEEvaluation::evaluate(values|gradients) for one component of one cell
  inline void evaluate(const Geometry &geo, const double *u_local, double *val, V3 *grad)
  {
    for (int q = 0; q < geo.nq; ++q)
      {
        double v = 0.0;
        V3     g;
        for (int l = 0; l < geo.nq; ++l)
          {
            v += geo.shape[q][l] * u_local[l];
            for (int d = 0; d < 3; ++d)
              g[d] += geo.dshape[q][l][d] * u_local[l];
          }
        val[q]  = v;
        grad[q] = g;
      }
  }

  // FEEvaluation::integrate(values|gradients) for one component of one cell:
  // r_l = sum_q JxW (v_q phi_l(q) + g_q . grad phi_l(q))
  inline void integrate(const Geometry &geo, const double *val, const V3 *grad, double *r_local)
  {
    for (int l = 0; l < geo.nq; ++l)
      {
        double r = 0.0;
        for (int q = 0; q < geo.nq; ++q)
          r += geo.JxW * (val[q] * geo.shape[q][l] + dot(grad[q], V3{{geo.dshape[q][l][0], geo.dshape[q][l][1],
                                                                       geo.dshape[q][l][2]}}));
        r_local[l] = r;
      }
  }

  inline int check_args(const oracle_mesh *m, const oracle_params *p)
  {
    if (!m || !p)
      return 1;
    if (m->dim != 2 && m->dim != 3)
      return 1;
    if (p->n_grains < 1 || p->n_grains > MAXG)
      return 2;
    for (int d = 0; d < m->dim; ++d)
      if (m->n[d] < 1 || !(m->h[d] > 0.0))
        return 1;
    return 0;
  }

  inline Mobility make_mobility(const oracle_mesh *m, const oracle_params *p)
  {
    return Mobility{m->dim, p->Mvol, p->Mvap, p->Msurf, p->Mgb, p->L, p->tensorial != 0};
  }

  // Advection velocity of grain b at quadrature point q of cell (i,j,k); false
  // when the cell belongs to no segment of b (AdvectionVelocityData::
  // has_velocity / get_velocity, sintering/advection.h:225-263).
  inline bool advection_velocity(const oracle_advection *a, const Geometry &geo, int b, int i, int j, int k, int q,
                                 V3 &v)
  {
    if (!a)
      return false;
    const int64_t cell = int64_t(i) + int64_t(geo.n[0]) * (int64_t(j) + int64_t(geo.n[1]) * k);
    const int     s    = a->cell_segments[int64_t(b) * geo.n_cells + cell];
    if (s < 0)
      return false;
    const double *d     = a->segments + 9 * int64_t(s);
    const double  gp[2] = {0.5 - 0.5 / std::sqrt(3.0), 0.5 + 0.5 / std::sqrt(3.0)};
    const int     co[3] = {i, j, k};
    double        r[3]  = {0.0, 0.0, 0.0};
    for (int e = 0; e < geo.dim; ++e)
      r[e] = a->origin[e] + (co[e] + gp[(q >> e) & 1]) * geo.h[e] - d[6 + e];
    // v_t + w x r
    v[0] = d[0] + d[4] * r[2] - d[5] * r[1];
    v[1] = d[1] + d[5] * r[0] - d[3] * r[2];
    v[2] = geo.dim == 3 ? d[2] + d[3] * r[1] - d[4] * r[0] : 0.0;
    return true;
  }

  // Blocks cell (i,j,k) works on: blk[0] = c, blk[1] = mu, blk[2..] = the
  // relevant grains' blocks in increasing order (all grains without a mask).
  // Returns the number of relevant grains.
  inline int cell_blocks(const Geometry &geo, const uint16_t *mask, int G, int i, int j, int k, int *blk)
  {
    blk[0] = 0;
    blk[1] = 1;
    const unsigned m =
      mask ? mask[int64_t(i) + int64_t(geo.n[0]) * (int64_t(j) + int64_t(geo.n[1]) * k)] : 0xffffffffu;
    int n = 0;
    for (int b = 0; b < G; ++b)
      if ((m >> b) & 1u)
        blk[2 + n++] = 2 + b;
    return n;
  }
}

extern "C" {

// free_energy.h:111-168 at one state (c, mu, eta_1..eta_G).  out receives
// f, df_dc, df_detai[G], d2f_dc2, d2f_dcdetai[G], d2f_detai2[G],
// d2f_detaidetaj[G*G] (row-major, i != j entries).
int oracle_free_energy(double A, double B, const double *state, int G, double *out)
{
  if (G < 1 || G > MAXG)
    return 2;
  const FreeEnergyEval fe(A, B, state, G);
  int                  k = 0;
  out[k++]               = fe.f();
  out[k++]               = fe.df_dc();
  for (int i = 0; i < G; ++i)
    out[k++] = fe.df_detai(state[2 + i]);
  out[k++] = fe.d2f_dc2();
  for (int i = 0; i < G; ++i)
    out[k++] = fe.d2f_dcdetai(state[2 + i]);
  for (int i = 0; i < G; ++i)
    out[k++] = fe.d2f_detai2(state[2 + i]);
  for (int i = 0; i < G; ++i)
    for (int j = 0; j < G; ++j)
      out[k++] = i == j ? 0.0 : fe.d2f_detaidetaj(state[2 + i], state[2 + j]);
  return 0;
}

// SinteringOperatorData::set_component_mask (operator_sintering_data.h:149-203)
// per cell: bit b of mask[cell] is set when the l-infinity norm of the cell's
// nodal values of eta_b exceeds tol.  (The reference takes the union over the
// cells of one SIMD batch; the restatement keeps one set per cell.)
int oracle_grain_mask(const oracle_mesh *m, const oracle_params *p, const double *u, double tol, uint16_t *mask)
{
  if (int e = check_args(m, p))
    return e;
  if (!(tol >= 0.0))
    return 1;
  const Geometry geo(*m);
  const int      G  = p->n_grains;
  const int64_t  N  = geo.n_nodes;
  const int      nk = geo.dim == 3 ? geo.n[2] : 1;
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < geo.n[1]; ++j)
      for (int i = 0; i < geo.n[0]; ++i)
        {
          unsigned bits = 0;
          for (int b = 0; b < G; ++b)
            {
              double norm = 0.0;
              for (int l = 0; l < geo.nq; ++l)
                norm = std::max(norm, std::fabs(u[(2 + b) * N + geo.node(i, j, k, l)]));
              if (norm > tol)
                bits |= 1u << b;
            }
          mask[int64_t(i) + int64_t(geo.n[0]) * (int64_t(j) + int64_t(geo.n[1]) * k)] = uint16_t(bits);
        }
  return 0;
}

// numerics/power_helper.h:31-45: sum_i x_i^p
double oracle_power_sum(const double *x, int n, int p)
{
  double s = 0.0;
  for (int i = 0; i < n; ++i)
    {
      double t = 1.0;
      for (int k = 0; k < p; ++k)
        t *= x[i];
      s += t;
    }
  return s;
}

// Nonlinear residual R(u):
//   SinteringOperatorGeneric::evaluate_nonlinear_residual<with_td>
//   (sintering/operator_sintering_generic.h:393-448), cell loop :977-1006,
//   history :927-975, quadrature kernel :254-308.
// hist[i] (i < time->order) are the old solutions; the history term is
// sum_i w_hist[i] * hist[i], interpolated to the quadrature points.
// dst is overwritten.
int oracle_residual(const oracle_mesh *m, const oracle_params *p, const oracle_time *t, const double *u,
                    const double *const *hist, int with_td, const uint16_t *mask, const oracle_advection *adv,
                    double *dst, int n_threads)
{
  if (int e = check_args(m, p))
    return e;
  if (with_td < 0 || with_td > 2 || !t)
    return 1;
  if (with_td == 2 && (t->order < 1 || t->order > 4 || !hist))
    return 1;
  const Geometry geo(*m);
  const Mobility mob = make_mobility(m, p);
  const int      G = p->n_grains, C = G + 2, nq = geo.nq;
  const int64_t  N = geo.n_nodes;
  std::memset(dst, 0, sizeof(double) * C * N);

  coloured_cell_loop(geo, n_threads, [&](int i, int j, int k) {
    int       blk[MAXC];
    const int G = cell_blocks(geo, mask, p->n_grains, i, j, k, blk), C = G + 2;
    double    ul[MAXC][8], hl[MAXC][8];
    double    val[MAXC][8], hval[MAXC][8];
    V3        grad[MAXC][8];
    for (int l = 0; l < nq; ++l)
      {
        const int64_t gi = geo.node(i, j, k, l);
        for (int b = 0; b < C; ++b)
          {
            ul[b][l] = u[blk[b] * N + gi];
            if (with_td == 2)
              {
                // generic.h:947-966: weighted sum of the old solutions at the nodes
                double s = 0.0;
                for (int o = 0; o < t->order; ++o)
                  s = (o == 0) ? hist[o][blk[b] * N + gi] * t->w_hist[o]
                               : s + hist[o][blk[b] * N + gi] * t->w_hist[o];
                hl[b][l] = s;
              }
          }
      }
    for (int b = 0; b < C; ++b)
      {
        evaluate(geo, ul[b], val[b], grad[b]);
        if (with_td == 2)
          {
            V3 dummy[8];
            evaluate(geo, hl[b], hval[b], dummy);
          }
      }
    double rv[MAXC][8];
    V3     rg[MAXC][8];
    for (int q = 0; q < nq; ++q)
      {
        double value[MAXC] = {};
        V3     gradient[MAXC];
        for (int b = 0; b < C; ++b)
          {
            value[b]    = val[b][q];
            gradient[b] = grad[b][q];
          }
        const double        *etas_value    = value + 2;
        const V3            *etas_gradient = gradient + 2;
        const FreeEnergyEval fe(p->A, p->B, value, G);
        // generic.h:274-285 c row
        double vr0 = 0.0;
        if (with_td >= 1)
          vr0 = value[0] * t->w0;
        if (with_td == 2)
          vr0 += hval[0][q];
        rv[0][q] = vr0;
        rg[0][q] = mob.apply_M(value[0], etas_value, G, gradient[0], etas_gradient, gradient[1]);
        // generic.h:287-289 mu row
        rv[1][q] = t->w_alg * value[1] - fe.df_dc();
        rg[1][q] = (-p->kappa_c) * gradient[0];
        // generic.h:292-304 eta rows
        for (int ig = 0; ig < G; ++ig)
          {
            double v = p->L * fe.df_detai(etas_value[ig]);
            if (with_td >= 1)
              v += value[ig + 2] * t->w0;
            if (with_td == 2)
              v += hval[2 + ig][q];
            rv[2 + ig][q] = v;
            rg[2 + ig][q] = (p->L * p->kappa_p) * gradient[2 + ig];
          }
        // generic.h:1015-1036: advection of c and eta_i with grain i's velocity
        for (int ig = 0; ig < G; ++ig)
          {
            V3 vel;
            if (advection_velocity(adv, geo, blk[2 + ig] - 2, i, j, k, q, vel))
              {
                rg[0][q]      = rg[0][q] - vel * value[0];
                rg[2 + ig][q] = rg[2 + ig][q] - vel * value[2 + ig];
              }
          }
      }
    for (int b = 0; b < C; ++b)
      {
        double rl[8];
        integrate(geo, rv[b], rg[b], rl);
        for (int l = 0; l < nq; ++l)
          dst[blk[b] * N + geo.node(i, j, k, l)] += rl[l];
      }
  });
  return 0;
}

// Jacobian-vector product J(lin) * src:
//   SinteringOperatorGeneric::vmult -> do_vmult_range (generic.h:539-577),
//   quadrature kernel SinteringOperatorGenericQuad (generic.h:101-190).
// The linearisation point is evaluated from the nodal vector `lin` (what
// fill_quadrature_point_values caches, operator_sintering_data.h:300-409).
// No constrained DoFs exist on these meshes (operator_base.h:294-353 is then
// a plain cell loop).  dst is overwritten.
int oracle_jvp(const oracle_mesh *m, const oracle_params *p, const oracle_time *t, const double *lin,
               const double *src, const uint16_t *mask, const oracle_advection *adv, double *dst, int n_threads)
{
  if (int e = check_args(m, p))
    return e;
  if (!t)
    return 1;
  const Geometry geo(*m);
  const Mobility mob = make_mobility(m, p);
  const int      G = p->n_grains, C = G + 2, nq = geo.nq;
  const int64_t  N = geo.n_nodes;
  std::memset(dst, 0, sizeof(double) * C * N);

  coloured_cell_loop(geo, n_threads, [&](int i, int j, int k) {
    int       blk[MAXC];
    const int G = cell_blocks(geo, mask, p->n_grains, i, j, k, blk), C = G + 2;
    double    ll[MAXC][8], sl[MAXC][8];
    double    lval[MAXC][8], sval[MAXC][8];
    V3        lgrad[MAXC][8], sgrad[MAXC][8];
    for (int l = 0; l < nq; ++l)
      {
        const int64_t gi = geo.node(i, j, k, l);
        for (int b = 0; b < C; ++b)
          {
            ll[b][l] = lin[blk[b] * N + gi];
            sl[b][l] = src[blk[b] * N + gi];
          }
      }
    for (int b = 0; b < C; ++b)
      {
        evaluate(geo, ll[b], lval[b], lgrad[b]);
        evaluate(geo, sl[b], sval[b], sgrad[b]);
      }
    double rv[MAXC][8];
    V3     rg[MAXC][8];
    for (int q = 0; q < nq; ++q)
      {
        double lin_value[MAXC] = {}, value[MAXC] = {};
        V3     lin_gradient[MAXC], gradient[MAXC];
        for (int b = 0; b < C; ++b)
          {
            lin_value[b]    = lval[b][q];
            lin_gradient[b] = lgrad[b][q];
            value[b]        = sval[b][q];
            gradient[b]     = sgrad[b][q];
          }
        const double        *lin_etas = lin_value + 2;
        const FreeEnergyEval fe(p->A, p->B, lin_value, G);
        double               value_result[MAXC] = {0.0};
        V3                   gradient_result[MAXC];
        // generic.h:120-134 c row
        value_result[0]    = value[0] * t->w0;
        gradient_result[0] = mob.apply_M_derivative(lin_value, lin_gradient, G, value, gradient);
        // generic.h:138-146 mu row
        value_result[1] = t->w_alg * value[1] - fe.d2f_dc2() * value[0];
        for (int ig = 0; ig < G; ++ig)
          value_result[1] -= fe.d2f_dcdetai(lin_etas[ig]) * value[ig + 2];
        gradient_result[1] = (-p->kappa_c) * gradient[0];
        // generic.h:150-163 eta rows
        for (int ig = 0; ig < G; ++ig)
          {
            value_result[ig + 2] += value[ig + 2] * t->w0 +
                                    p->L * (fe.d2f_dcdetai(lin_etas[ig]) * value[0] +
                                            fe.d2f_detai2(lin_etas[ig]) * value[ig + 2]);
            gradient_result[ig + 2] = (p->L * p->kappa_p) * gradient[ig + 2];
          }
        apply_d2f_detaidetaj(p->B, p->L, lin_etas, G, value + 2, value_result + 2);
        // generic.h:167-177: advection with the (frozen) grain velocities
        for (int ig = 0; ig < G; ++ig)
          {
            V3 vel;
            if (advection_velocity(adv, geo, blk[2 + ig] - 2, i, j, k, q, vel))
              {
                gradient_result[0]      = gradient_result[0] - vel * value[0];
                gradient_result[ig + 2] = gradient_result[ig + 2] - vel * value[ig + 2];
              }
          }
        for (int b = 0; b < C; ++b)
          {
            rv[b][q] = value_result[b];
            rg[b][q] = gradient_result[b];
          }
      }
    for (int b = 0; b < C; ++b)
      {
        double rl[8];
        integrate(geo, rv[b], rg[b], rl);
        for (int l = 0; l < nq; ++l)
          dst[blk[b] * N + geo.node(i, j, k, l)] += rl[l];
      }
  });
  return 0;
}

// Diagonal of the Allen-Cahn block operator (G blocks of N, not inverted):
//   OperatorAllenCahn::do_vmult_kernel (sintering/preconditioners.h:342-414)
//   assembled by MatrixFreeTools::compute_diagonal as in
//   OperatorBase::compute_inverse_diagonal (operator_base.h:364-389).
// The unit vector e_(node,grain) only excites value[ig]; the eta_i-eta_j
// coupling lands off the diagonal, so
//   d_i(n) = sum_cells sum_q JxW [(w0 + L f_{eta_i eta_i}) phi_n^2 + L kappa_p |grad phi_n|^2].
int oracle_ac_diagonal(const oracle_mesh *m, const oracle_params *p, const oracle_time *t, const double *lin,
                       const uint16_t *mask, const oracle_advection *adv, double *diag, int n_threads)
{
  if (int e = check_args(m, p))
    return e;
  const Geometry geo(*m);
  const int      G = p->n_grains, nq = geo.nq;
  const int64_t  N = geo.n_nodes;
  std::memset(diag, 0, sizeof(double) * G * N);
  coloured_cell_loop(geo, n_threads, [&](int i, int j, int k) {
    // cut-off: absent grains add nothing (preconditioners.h:787-817)
    int       blk[MAXC];
    const int G = cell_blocks(geo, mask, p->n_grains, i, j, k, blk), C = G + 2;
    double    ll[MAXC][8], lval[MAXC][8];
    V3        lgrad[MAXC][8];
    for (int l = 0; l < nq; ++l)
      for (int b = 0; b < C; ++b)
        ll[b][l] = lin[blk[b] * N + geo.node(i, j, k, l)];
    for (int b = 0; b < C; ++b)
      evaluate(geo, ll[b], lval[b], lgrad[b]);
    for (int ig = 0; ig < G; ++ig)
      for (int l = 0; l < nq; ++l)
        {
          double d = 0.0;
          for (int q = 0; q < nq; ++q)
            {
              double lv[MAXC];
              for (int b = 0; b < C; ++b)
                lv[b] = lval[b][q];
              const FreeEnergyEval fe(p->A, p->B, lv, G);
              const double         phi = geo.shape[q][l];
              const V3             dphi{{geo.dshape[q][l][0], geo.dshape[q][l][1], geo.dshape[q][l][2]}};
              const double         vr  = phi * t->w0 + p->L * fe.d2f_detai2(lv[2 + ig]) * phi;
              V3                   gr  = (p->L * p->kappa_p) * dphi;
              // precondition_advection_ac (operator_sintering_generic.h:826-850),
              // each grain with its own velocity and its own trial function
              V3 vel;
              if (advection_velocity(adv, geo, blk[2 + ig] - 2, i, j, k, q, vel))
                gr = gr - vel * phi;
              d += geo.JxW * (vr * phi + dot(gr, dphi));
            }
          diag[(blk[2 + ig] - 2) * N + geo.node(i, j, k, l)] += d;
        }
  });
  return 0;
}

// Node-diagonal 2x2 blocks of the Cahn-Hilliard tangent
//   OperatorCahnHilliard::do_vmult_kernel (sintering/preconditioners.h:85-169)
// restricted to (node n, node n):  blocks[0*N+n] = J_cc, [1*N+n] = J_c,mu,
// [2*N+n] = J_mu,c, [3*N+n] = J_mu,mu  (row = tested equation, col = unknown).
int oracle_ch_blocks(const oracle_mesh *m, const oracle_params *p, const oracle_time *t, const double *lin,
                     const uint16_t *mask, const oracle_advection *adv, double *blocks, int n_threads)
{
  if (int e = check_args(m, p))
    return e;
  const Geometry geo(*m);
  const Mobility mob = make_mobility(m, p);
  const int      nq  = geo.nq;
  const int64_t  N   = geo.n_nodes;
  std::memset(blocks, 0, sizeof(double) * 4 * N);
  coloured_cell_loop(geo, n_threads, [&](int i, int j, int k) {
    int       blk[MAXC];
    const int G = cell_blocks(geo, mask, p->n_grains, i, j, k, blk), C = G + 2;
    double    ll[MAXC][8], lval[MAXC][8];
    V3        lgrad[MAXC][8];
    for (int l = 0; l < nq; ++l)
      for (int b = 0; b < C; ++b)
        ll[b][l] = lin[blk[b] * N + geo.node(i, j, k, l)];
    for (int b = 0; b < C; ++b)
      evaluate(geo, ll[b], lval[b], lgrad[b]);
    for (int l = 0; l < nq; ++l)
      {
        double J[4] = {0, 0, 0, 0};
        for (int q = 0; q < nq; ++q)
          {
            double lv[MAXC];
            V3     lg[MAXC];
            for (int b = 0; b < C; ++b)
              {
                lv[b] = lval[b][q];
                lg[b] = lgrad[b][q];
              }
            const double         c = lv[0];
            const V3            &c_grad = lg[0], &mu_grad = lg[1];
            const FreeEnergyEval fe(p->A, p->B, lv, G);
            const double         phi = geo.shape[q][l];
            const V3             dphi{{geo.dshape[q][l][0], geo.dshape[q][l][1], geo.dshape[q][l][2]}};
            // unknown c: value = phi, gradient = dphi (mu = 0)
            {
              const double vr0 = phi * t->w0;
              const double vr1 = -fe.d2f_dc2() * phi;
              V3 gr0 = mul(mob.dM_dc(c, c_grad), mu_grad) * phi + mul(mob.dM_dgrad_c(c, c_grad, mu_grad), dphi);
              const V3     gr1 = (-p->kappa_c) * dphi;
              // precondition_advection_ch (operator_sintering_generic.h:800-824)
              for (int ig = 0; ig < G; ++ig)
                {
                  V3 vel;
                  if (advection_velocity(adv, geo, blk[2 + ig] - 2, i, j, k, q, vel))
                    gr0 = gr0 - vel * phi;
                }
              J[0] += geo.JxW * (vr0 * phi + dot(gr0, dphi));
              J[2] += geo.JxW * (vr1 * phi + dot(gr1, dphi));
            }
            // unknown mu: value = phi, gradient = dphi (c = 0)
            {
              const double vr1 = phi * t->w_alg;
              const V3     gr0 = mob.apply_M(c, lv + 2, G, c_grad, lg + 2, dphi);
              J[1] += geo.JxW * dot(gr0, dphi);
              J[3] += geo.JxW * (vr1 * phi);
            }
          }
        const int64_t gi = geo.node(i, j, k, l);
        for (int e = 0; e < 4; ++e)
          blocks[e * N + gi] += J[e];
      }
  });
  return 0;
}

// Assembled Cahn-Hilliard block of the tangent, the matrix hpsint builds for
// its matrix-based CH preconditioner (MyMatrixFreeTools::compute_matrix,
// matrix_free/tools.h:29-175, on OperatorCahnHilliard::do_vmult_kernel,
// sintering/preconditioners.h:85-169, set up by BlockPreconditioner2::
// do_update, preconditioners.h:1260-1283).  Stored by node row as 2x2 blocks
// for each of the 3^dim neighbours: A[(k * 4 + e) * N + n] with neighbour
// k = (dx + 1) + 3 (dy + 1) (+ 9 (dz + 1)) of node n and entry e = 0 J_cc,
// 1 J_c,mu, 2 J_mu,c, 3 J_mu,mu (row = tested equation, column = unknown).
// The trial functions of the columns enter exactly as in oracle_ch_blocks,
// whose values are the k = centre blocks.
int oracle_ch_matrix(const oracle_mesh *m, const oracle_params *p, const oracle_time *t, const double *lin,
                     const uint16_t *mask, const oracle_advection *adv, double *A, int n_threads)
{
  if (int e = check_args(m, p))
    return e;
  const Geometry geo(*m);
  const Mobility mob = make_mobility(m, p);
  const int      nq  = geo.nq, NK = geo.dim == 3 ? 27 : 9;
  const int64_t  N   = geo.n_nodes;
  std::memset(A, 0, sizeof(double) * NK * 4 * N);
  coloured_cell_loop(geo, n_threads, [&](int i, int j, int k) {
    int       blk[MAXC];
    const int G = cell_blocks(geo, mask, p->n_grains, i, j, k, blk), C = G + 2;
    double    ll[MAXC][8], lval[MAXC][8];
    V3        lgrad[MAXC][8];
    for (int l = 0; l < nq; ++l)
      for (int b = 0; b < C; ++b)
        ll[b][l] = lin[blk[b] * N + geo.node(i, j, k, l)];
    for (int b = 0; b < C; ++b)
      evaluate(geo, ll[b], lval[b], lgrad[b]);
    for (int l = 0; l < nq; ++l)
      for (int mm = 0; mm < nq; ++mm)
        {
          double J[4] = {0, 0, 0, 0};
          for (int q = 0; q < nq; ++q)
            {
              double lv[MAXC];
              V3     lg[MAXC];
              for (int b = 0; b < C; ++b)
                {
                  lv[b] = lval[b][q];
                  lg[b] = lgrad[b][q];
                }
              const double         c = lv[0];
              const V3            &c_grad = lg[0], &mu_grad = lg[1];
              const FreeEnergyEval fe(p->A, p->B, lv, G);
              const double         phi = geo.shape[q][l], psi = geo.shape[q][mm];
              const V3 dphi{{geo.dshape[q][l][0], geo.dshape[q][l][1], geo.dshape[q][l][2]}};
              const V3 dpsi{{geo.dshape[q][mm][0], geo.dshape[q][mm][1], geo.dshape[q][mm][2]}};
              // unknown c: value = psi, gradient = dpsi (mu = 0)
              {
                const double vr0 = psi * t->w0;
                const double vr1 = -fe.d2f_dc2() * psi;
                V3 gr0 = mul(mob.dM_dc(c, c_grad), mu_grad) * psi + mul(mob.dM_dgrad_c(c, c_grad, mu_grad), dpsi);
                const V3 gr1 = (-p->kappa_c) * dpsi;
                for (int ig = 0; ig < G; ++ig)
                  {
                    V3 vel;
                    if (advection_velocity(adv, geo, blk[2 + ig] - 2, i, j, k, q, vel))
                      gr0 = gr0 - vel * psi;
                  }
                J[0] += geo.JxW * (vr0 * phi + dot(gr0, dphi));
                J[2] += geo.JxW * (vr1 * phi + dot(gr1, dphi));
              }
              // unknown mu: value = psi, gradient = dpsi (c = 0)
              {
                const double vr1 = psi * t->w_alg;
                const V3     gr0 = mob.apply_M(c, lv + 2, G, c_grad, lg + 2, dpsi);
                J[1] += geo.JxW * dot(gr0, dphi);
                J[3] += geo.JxW * (vr1 * phi);
              }
            }
          const int dx = (mm & 1) - (l & 1), dy = ((mm >> 1) & 1) - ((l >> 1) & 1),
                    dz = geo.dim == 3 ? ((mm >> 2) & 1) - ((l >> 2) & 1) : 0;
          const int     kk = (dx + 1) + 3 * (dy + 1) + (geo.dim == 3 ? 9 * (dz + 1) : 0);
          const int64_t gi = geo.node(i, j, k, l);
          for (int e = 0; e < 4; ++e)
            A[(int64_t(kk) * 4 + e) * N + gi] += J[e];
        }
  });
  return 0;
}

namespace
{
  // 2x2 inverse of a node's centre block, guarded as the block-Jacobi
  // preconditioner's: a singular block falls back to the guarded point
  // inverse of its diagonal (operator_base.h:386-388).
  inline void invert_2x2(double a, double b, double c, double d, double inv[4])
  {
    const double det   = a * d - b * c;
    const double scale = std::fabs(a * d) + std::fabs(b * c);
    if (det != 0.0 && std::isfinite(det) && std::fabs(det) > 1e-14 * scale)
      {
        inv[0] = d / det;
        inv[1] = -b / det;
        inv[2] = -c / det;
        inv[3] = a / det;
      }
    else
      {
        inv[0] = std::fabs(a) > 1.0e-10 ? 1.0 / a : 1.0;
        inv[3] = std::fabs(d) > 1.0e-10 ? 1.0 / d : 1.0;
        inv[1] = inv[2] = 0.0;
      }
  }
} // namespace

// Symmetric Gauss-Seidel preconditioner of the assembled CH block in
// multicolour order: z = M^-1 r with M = (D + L) D^-1 (D + U), where nodes are
// ordered by colour (parity of the node index in each direction: 2^dim
// colours, no two nodes of one colour share a cell) and D holds the 2x2
// centre blocks.  Forward sweep, colours ascending:
//   y_n = D_n^-1 (r_n - sum_{j, colour(j) < colour(n)} A_nj y_j),
// backward sweep, colours descending from the second-last:
//   z_n = y_n - D_n^-1 sum_{j, colour(j) > colour(n)} A_nj z_j.
// Neighbours are summed in the order k = 0 .. 3^dim - 1.  r and z: 2 x N.
int oracle_ch_sgs(const oracle_mesh *m, const double *A, const double *r, double *z)
{
  if (!m || !A || !r || !z)
    return 1;
  const Geometry geo(*m);
  const int      NK = geo.dim == 3 ? 27 : 9, n_col = 1 << geo.dim;
  const int64_t  N  = geo.n_nodes;
  std::vector<double> y(2 * N);
  auto colour = [&](int x, int yy, int zz) { return (x & 1) | ((yy & 1) << 1) | ((zz & 1) << 2); };
  auto sweep  = [&](int col, bool forward) {
    for (int kz = 0; kz < geo.nn[2]; ++kz)
      for (int ky = 0; ky < geo.nn[1]; ++ky)
        for (int kx = 0; kx < geo.nn[0]; ++kx)
          {
            if (colour(kx, ky, kz) != col)
              continue;
            const int64_t n = kx + int64_t(geo.nn[0]) * (ky + int64_t(geo.nn[1]) * kz);
            double        s0 = 0.0, s1 = 0.0;
            for (int k = 0; k < NK; ++k)
              {
                const int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = geo.dim == 3 ? k / 9 - 1 : 0;
                const int x = kx + dx, yy = ky + dy, zz = kz + dz;
                if (x < 0 || yy < 0 || zz < 0 || x >= geo.nn[0] || yy >= geo.nn[1] || zz >= geo.nn[2])
                  continue;
                const int cj = colour(x, yy, zz);
                if (forward ? !(cj < col) : !(cj > col))
                  continue;
                const int64_t j  = x + int64_t(geo.nn[0]) * (yy + int64_t(geo.nn[1]) * zz);
                const double *v  = forward ? y.data() : z;
                const double  v0 = v[j], v1 = v[N + j];
                s0 += A[(int64_t(k) * 4 + 0) * N + n] * v0 + A[(int64_t(k) * 4 + 1) * N + n] * v1;
                s1 += A[(int64_t(k) * 4 + 2) * N + n] * v0 + A[(int64_t(k) * 4 + 3) * N + n] * v1;
              }
            const int ctr = NK / 2;
            double    inv[4];
            invert_2x2(A[(int64_t(ctr) * 4 + 0) * N + n], A[(int64_t(ctr) * 4 + 1) * N + n],
                       A[(int64_t(ctr) * 4 + 2) * N + n], A[(int64_t(ctr) * 4 + 3) * N + n], inv);
            if (forward)
              {
                const double a0 = r[n] - s0, a1 = r[N + n] - s1;
                y[n]            = inv[0] * a0 + inv[1] * a1;
                y[N + n]        = inv[2] * a0 + inv[3] * a1;
              }
            else
              {
                z[n]     = y[n] - (inv[0] * s0 + inv[1] * s1);
                z[N + n] = y[N + n] - (inv[2] * s0 + inv[3] * s1);
              }
          }
  };
  for (int col = 0; col < n_col; ++col)
    sweep(col, true);
  std::memcpy(z, y.data(), sizeof(double) * 2 * N);
  for (int col = n_col - 2; col >= 0; --col)
    sweep(col, false);
  return 0;
}

// GrainTracker particle detection for one order parameter on one process:
// run_flooding / detect_local_particle_groups
// (grain_tracker/distributed_stitching.h:41-100, :441-480).  A cell belongs
// to a particle when the largest of its nodal values exceeds threshold_lower;
// particles are the face-connected sets of such cells, numbered in the order
// the lexicographic cell loop (x fastest) first reaches them.  ids[cell] =
// particle number or -1; *n_particles = their number.
int oracle_grain_segments(const oracle_mesh *m, const double *eta, double threshold_lower, int *ids,
                          int *n_particles)
{
  if (!m || (m->dim != 2 && m->dim != 3) || !eta || !ids || !n_particles)
    return 1;
  const Geometry geo(*m);
  const int64_t  nc = geo.n_cells;
  auto cell_max = [&](int64_t c) {
    const int i = int(c % geo.n[0]), j = int((c / geo.n[0]) % geo.n[1]), k = int(c / (int64_t(geo.n[0]) * geo.n[1]));
    double mx = -std::numeric_limits<double>::infinity();
    for (int l = 0; l < geo.nq; ++l)
      mx = std::max(mx, eta[geo.node(i, j, k, l)]);
    return mx;
  };
  std::vector<char> flag(nc);
  for (int64_t c = 0; c < nc; ++c)
    {
      flag[c] = cell_max(c) > threshold_lower;
      ids[c]  = -1;
    }
  const int64_t stride[3] = {1, geo.n[0], int64_t(geo.n[0]) * geo.n[1]};
  int           count     = 0;
  std::vector<int64_t> stack;
  for (int64_t c0 = 0; c0 < nc; ++c0)
    {
      if (!flag[c0] || ids[c0] >= 0)
        continue;
      ids[c0] = count;
      stack.assign(1, c0);
      while (!stack.empty())
        {
          const int64_t c = stack.back();
          stack.pop_back();
          const int co[3] = {int(c % geo.n[0]), int((c / geo.n[0]) % geo.n[1]),
                             int(c / (int64_t(geo.n[0]) * geo.n[1]))};
          for (int d = 0; d < geo.dim; ++d)
            for (int s = -1; s <= 1; s += 2)
              {
                const int cd = co[d] + s;
                if (cd < 0 || cd >= geo.n[d])
                  continue; // cell->at_boundary(face)
                const int64_t nb = c + s * stride[d];
                if (flag[nb] && ids[nb] < 0)
                  {
                    ids[nb] = count;
                    stack.push_back(nb);
                  }
              }
        }
      ++count;
    }
  *n_particles = count;
  return 0;
}

// Particle properties of the spherical representation, per particle
// [measure, center[dim], radius, max value]: compute_particles_info
// (distributed_stitching.h:264-320: measure-weighted cell centers),
// compute_particles_radii (:322-360: max over the cells of the distance from
// the center to the cell's barycenter plus half its diameter) and the
// particle maxima of run_flooding (:77-86).  origin = lower corner of the mesh.
int oracle_segment_properties(const oracle_mesh *m, const double *origin, const double *eta, const int *ids,
                              int n_particles, double *props)
{
  if (!m || (m->dim != 2 && m->dim != 3) || !origin || !eta || !ids || !props || n_particles < 0)
    return 1;
  const Geometry geo(*m);
  const int      dim = geo.dim, nf = 3 + dim;
  double         vol = 1.0, diam2 = 0.0;
  for (int d = 0; d < dim; ++d)
    {
      vol *= geo.h[d];
      diam2 += geo.h[d] * geo.h[d];
    }
  const double        half_diam = 0.5 * std::sqrt(diam2);
  std::vector<double> sum(int64_t(n_particles) * (1 + dim), 0.0);
  for (int p = 0; p < n_particles; ++p)
    {
      props[p * nf + 1 + dim] = 0.0;
      props[p * nf + 2 + dim] = -std::numeric_limits<double>::infinity();
    }
  auto center_of = [&](int64_t c, double *x) {
    const int co[3] = {int(c % geo.n[0]), int((c / geo.n[0]) % geo.n[1]), int(c / (int64_t(geo.n[0]) * geo.n[1]))};
    for (int d = 0; d < dim; ++d)
      x[d] = origin[d] + (co[d] + 0.5) * geo.h[d];
  };
  for (int64_t c = 0; c < geo.n_cells; ++c)
    {
      const int p = ids[c];
      if (p < 0)
        continue;
      if (p >= n_particles)
        return 1;
      double x[3];
      center_of(c, x);
      sum[int64_t(p) * (1 + dim)] += vol;
      for (int d = 0; d < dim; ++d)
        sum[int64_t(p) * (1 + dim) + 1 + d] += x[d] * vol;
      const int i = int(c % geo.n[0]), j = int((c / geo.n[0]) % geo.n[1]), k = int(c / (int64_t(geo.n[0]) * geo.n[1]));
      for (int l = 0; l < geo.nq; ++l)
        props[p * nf + 2 + dim] = std::max(props[p * nf + 2 + dim], eta[geo.node(i, j, k, l)]);
    }
  for (int p = 0; p < n_particles; ++p)
    {
      props[p * nf] = sum[int64_t(p) * (1 + dim)];
      for (int d = 0; d < dim; ++d)
        props[p * nf + 1 + d] = sum[int64_t(p) * (1 + dim) + 1 + d] / sum[int64_t(p) * (1 + dim)];
    }
  for (int64_t c = 0; c < geo.n_cells; ++c)
    {
      const int p = ids[c];
      if (p < 0)
        continue;
      double x[3], r2 = 0.0;
      center_of(c, x);
      for (int d = 0; d < dim; ++d)
        r2 += (x[d] - props[p * nf + 1 + d]) * (x[d] - props[p * nf + 1 + d]);
      props[p * nf + 1 + dim] = std::max(props[p * nf + 1 + dim], std::sqrt(r2) + half_diam);
    }
  return 0;
}

// AdvectionOperatorGeneric::evaluate_forces / do_evaluate_forces
// (sintering/operator_advection.h:86-373): for every cell and every relevant
// grain i whose order parameter has a segment s on the cell, with the
// quadrature points x_q of the cell,
//   volume_s += sum_q eta_i JxW
//   force_s  += sum_q sum_{j != i relevant} dF_ij JxW,
//               dF_ij = k (c - ceq) f(eta_i eta_j) (grad eta_i - grad eta_j)
//   torque_s += sum_q sum_j (x_q - center_s) x dF_ij JxW
// with f(p) = 1 / (1 + exp(-smoothening (p - cgb))) (cgb > 0, smoothening
// > 0), [p > cgb] (cgb > 0) or 4 p (cgb <= 0), and hpsint's cross products
// (include/pf-applications/base/tensor.h:62-84: in 2D the scalar
// a[1] b[0] - a[0] b[1]).  out: n_segments rows of 1 + dim + (dim == 3 ? 3 :
// 1) values (volume, force, torque), overwritten; cells in lexicographic
// order, grains in increasing order.  centers: n_segments x 3.
int oracle_advection_forces(const oracle_mesh *m, const oracle_params *p, const double *origin, const double *u,
                            const uint16_t *mask, const int *cell_segments, const double *centers, int n_segments,
                            double k_stiff, double cgb, double ceq, double smoothening, double *out)
{
  if (int e = check_args(m, p))
    return e;
  if (!origin || !u || !cell_segments || n_segments < 0 || (n_segments > 0 && (!centers || !out)))
    return 1;
  const Geometry geo(*m);
  const int      dim = geo.dim, nt = dim == 3 ? 3 : 1, nc = 1 + dim + nt, nq = geo.nq;
  const int64_t  N = geo.n_nodes;
  std::fill(out, out + int64_t(n_segments) * nc, 0.0);
  const double gp[2] = {0.5 - 0.5 / std::sqrt(3.0), 0.5 + 0.5 / std::sqrt(3.0)};
  for (int k = 0; k < geo.n[2]; ++k)
    for (int j = 0; j < geo.n[1]; ++j)
      for (int i = 0; i < geo.n[0]; ++i)
        {
          const int64_t cell = int64_t(i) + int64_t(geo.n[0]) * (int64_t(j) + int64_t(geo.n[1]) * k);
          int           blk[MAXC];
          const int     G = cell_blocks(geo, mask, p->n_grains, i, j, k, blk), C = G + 2;
          double        val[MAXC][8];
          V3            grad[MAXC][8];
          for (int b = 0; b < C; ++b)
            {
              double ul[8];
              for (int l = 0; l < nq; ++l)
                ul[l] = u[blk[b] * N + geo.node(i, j, k, l)];
              evaluate(geo, ul, val[b], grad[b]);
            }
          const int co[3] = {i, j, k};
          for (int ig = 0; ig < G; ++ig)
            {
              const int s = cell_segments[int64_t(blk[2 + ig] - 2) * geo.n_cells + cell];
              if (s < 0)
                continue;
              if (s >= n_segments)
                return 1;
              double *o = out + int64_t(s) * nc;
              for (int q = 0; q < nq; ++q)
                {
                  double r[3] = {0.0, 0.0, 0.0};
                  for (int e = 0; e < dim; ++e)
                    r[e] = origin[e] + (co[e] + gp[(q >> e) & 1]) * geo.h[e] - centers[3 * int64_t(s) + e];
                  const double c = val[0][q], ei = val[2 + ig][q];
                  double       force[3] = {0.0, 0.0, 0.0}, torque[3] = {0.0, 0.0, 0.0};
                  for (int jg = 0; jg < G; ++jg)
                    {
                      if (jg == ig)
                        continue;
                      double f = ei * val[2 + jg][q];
                      if (cgb > 0.0)
                        f = smoothening > 0.0 ? 1.0 / (1.0 + std::exp(-smoothening * (f - cgb))) : (f > cgb ? 1.0 : 0.0);
                      else
                        f *= 4.0;
                      const double w = k_stiff * (c - ceq) * f;
                      double       dF[3];
                      for (int e = 0; e < 3; ++e)
                        dF[e] = (grad[2 + ig][q][e] - grad[2 + jg][q][e]) * w;
                      for (int e = 0; e < dim; ++e)
                        force[e] += dF[e];
                      if (dim == 3)
                        {
                          torque[0] += r[1] * dF[2] - r[2] * dF[1];
                          torque[1] += r[2] * dF[0] - r[0] * dF[2];
                          torque[2] += r[0] * dF[1] - r[1] * dF[0];
                        }
                      else
                        torque[0] += r[1] * dF[0] - r[0] * dF[1];
                    }
                  o[0] += ei * geo.JxW;
                  for (int e = 0; e < dim; ++e)
                    o[1 + e] += force[e] * geo.JxW;
                  for (int e = 0; e < nt; ++e)
                    o[1 + dim + e] += torque[e] * geo.JxW;
                }
            }
        }
  return 0;
}

// CFLChecker::check_courant (sintering/cfl_checker.h:62-128): returns 1 when
// |v| dt < cell diameter for every relevant grain with a velocity at every
// quadrature point of every cell, else 0 (-1 on bad arguments).
int oracle_advection_courant(const oracle_mesh *m, const oracle_params *p, const uint16_t *mask,
                             const oracle_advection *adv, double dt)
{
  if (check_args(m, p) || !adv)
    return -1;
  const Geometry geo(*m);
  double         diam2 = 0.0;
  for (int d = 0; d < geo.dim; ++d)
    diam2 += geo.h[d] * geo.h[d];
  const double diam = std::sqrt(diam2);
  for (int k = 0; k < geo.n[2]; ++k)
    for (int j = 0; j < geo.n[1]; ++j)
      for (int i = 0; i < geo.n[0]; ++i)
        {
          int       blk[MAXC];
          const int G = cell_blocks(geo, mask, p->n_grains, i, j, k, blk);
          for (int ig = 0; ig < G; ++ig)
            for (int q = 0; q < geo.nq; ++q)
              {
                V3 v;
                if (advection_velocity(adv, geo, blk[2 + ig] - 2, i, j, k, q, v) &&
                    !(std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * dt < diam))
                  return 0;
              }
        }
  return 1;
}

// AdvectionMechanism::calc_translation_velocity / calc_rotation_velocity
// (sintering/advection.h:330-352): per segment the velocity table the
// residual and J v read: v_t = mt force / volume, w = mr torque / volume (the
// z component in 2D, cross(r) = torque (-r[1], r[0]), advection.h:105-113),
// center.  A segment without volume gets no velocity.  vft: n_segments rows
// of 1 + dim + (dim == 3 ? 3 : 1) values; centers: n_segments x 3; segments:
// n_segments x 9 (overwritten).
int oracle_advection_velocities(int dim, const double *vft, const double *centers, int n_segments, double mt,
                                double mr, double *segments)
{
  if ((dim != 2 && dim != 3) || n_segments < 0 || (n_segments > 0 && (!vft || !centers || !segments)))
    return 1;
  const int nt = dim == 3 ? 3 : 1, nc = 1 + dim + nt;
  for (int s = 0; s < n_segments; ++s)
    {
      const double *d = vft + int64_t(s) * nc;
      double       *o = segments + 9 * int64_t(s);
      for (int e = 0; e < 9; ++e)
        o[e] = 0.0;
      for (int e = 0; e < 3; ++e)
        o[6 + e] = centers[3 * int64_t(s) + e];
      if (!(d[0] > 0.0))
        continue;
      for (int e = 0; e < dim; ++e)
        o[e] = mt * d[1 + e] / d[0];
      if (dim == 3)
        for (int e = 0; e < 3; ++e)
          o[3 + e] = mr * d[1 + dim + e] / d[0];
      else
        o[5] = mr * d[1 + dim] / d[0];
    }
  return 0;
}

} // extern "C"
