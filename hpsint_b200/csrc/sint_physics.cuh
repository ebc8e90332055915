// Point-wise physics of the sintering operator at one quadrature point.
//
// Restates, for Real = double or float and a compile-time number of grains G:
//   sintering/free_energy.h:111-168, :233-252     (Wang bulk energy)
//   sintering/mobility.h:439-534                  (MobilityScalar)
//   sintering/mobility.h:668-916, :960            (MobilityTensorial)
//   include/pf-applications/base/tensor.h:137-186 (unit_vector, filters, projector)
// Vectors are plain arrays of length DIM.  The grain-boundary pair loops keep
// hpsint's lower-triangular (i > j) order; algebraically equal terms that only
// depend on the linearisation point are grouped to save operations.
#pragma once

#include "sint_common.cuh"
#include <type_traits>

namespace sint
{
  // c ? a : b, written as a call so that the packed FP32 pairs (F2, whose
  // comparisons give one flag per lane) select lane by lane
  template <typename R>
  __device__ __forceinline__ R sel(bool c, R a, R b)
  {
    return c ? a : b;
  }

  template <int D, typename R>
  __device__ __forceinline__ R dotv(const R (&a)[D], const R (&b)[D])
  {
    R s = a[0] * b[0];
#pragma unroll
    for (int d = 1; d < D; ++d)
      s += a[d] * b[d];
    return s;
  }

  // Reciprocal and inverse square root of a positive number by Newton-Raphson
  // refinement of the single-precision hardware seed (rcp.approx /
  // rsqrt.approx, relative error ~2^-23 including the rounding of the
  // argument to float):
  //   reciprocal:          y <- y + y (1 - x y)
  //   inverse square root: y <- y + (y / 2) (1 - x y^2)
  // One step squares the relative error: ~3e-14 in double (far inside the
  // operator's 1e-12 parity bound), float rounding level in float.  The seeds
  // need the argument and the result inside the normal float range, [2^-126,
  // 2^126] for the reciprocal and [2^-126, 2^128) for the inverse square root.
  // In double the argument is scaled by 2^-56 before seeding and the result
  // back by the exact power of two, which moves that range to [2^-70, 2^182]
  // (8.5e-22 .. 6e54): the callers filter squared norms below 1e-20, and a
  // squared gradient norm above 6e54 would need a gradient steeper than
  // 2e27 per unit length.  (No branch: a guarded exact division here cost 8 %
  // of the FP64 Jacobian product.)
  __device__ __forceinline__ float rcp_seed(float x)
  {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
  }
  __device__ __forceinline__ float rsqrt_seed(float x)
  {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
  }

  template <typename R>
  __device__ __forceinline__ R seed_rcp(R x)
  {
    return R(rcp_seed(float(x)));
  }
  template <>
  __device__ __forceinline__ F2 seed_rcp<F2>(F2 x)
  {
    return F2(rcp_seed(x.v.x), rcp_seed(x.v.y));
  }
  template <typename R>
  __device__ __forceinline__ R seed_rsqrt(R x)
  {
    return R(rsqrt_seed(float(x)));
  }
  template <>
  __device__ __forceinline__ F2 seed_rsqrt<F2>(F2 x)
  {
    return F2(rsqrt_seed(x.v.x), rsqrt_seed(x.v.y));
  }

  template <typename R>
  __device__ __forceinline__ R rcp_pos(R x)
  {
    if constexpr (std::is_same_v<R, double>)
      {
        const double xs = x * 0x1p-56;
        const double s  = double(rcp_seed(float(xs)));
        return (s + s * (1.0 - xs * s)) * 0x1p-56;
      }
    else
      {
        const R y = seed_rcp(x);
        return y + y * (R(1) - x * y);
      }
  }

  template <typename R>
  __device__ __forceinline__ R rsqrt_pos(R x)
  {
    if constexpr (std::is_same_v<R, double>)
      {
        const double xs = x * 0x1p-56;
        const double s  = double(rsqrt_seed(float(xs)));
        return (s + (0.5 * s) * (1.0 - (xs * s) * s)) * 0x1p-28;
      }
    else
      {
        const R y = seed_rsqrt(x);
        return y + (R(0.5) * y) * (R(1) - (x * y) * y);
      }
  }

  template <typename R>
  __device__ __forceinline__ R clamp01(R x)
  {
    return fmin(fmax(x, R(0)), R(1));
  }
  __device__ __forceinline__ F2 clamp01(const P2 &x) { return clamp01(F2(x)); }

  // tensor.h:137-154 unit_vector(v, 1e-10): v / |v| if |v| > 1e-10, else 0.
  // Also returns n2 = |v|^2 and rs = 1 / |v| (0 below the threshold), which
  // the dM/dgrad c term reuses.
  template <int D, typename R>
  __device__ __forceinline__ void unit_vector(const R (&v)[D], R (&n)[D], R &n2, R &rs)
  {
    n2 = dotv<D>(v, v);
    // |v| > 1e-10  <=>  |v|^2 > 1e-20
    rs = sel(n2 > R(1e-20), rsqrt_pos<R>(n2), R(0));
#pragma unroll
    for (int d = 0; d < D; ++d)
      n[d] = v[d] * rs;
  }

  // tensor.h:156-174 unit_vector_filter_2(v, 1e-20): 1 / |v|^2 or 0
  template <int D, typename R>
  __device__ __forceinline__ R unit_vector_filter_2(const R (&v)[D])
  {
    const R n2 = dotv<D>(v, v);
    return sel(n2 > R(1e-20), rcp_pos<R>(n2), R(0));
  }

  // Grain cut-off (operator_sintering_data.h:149-203): bit i of the cell mask m
  // is set when grain i is relevant on the cell.  Absent grains enter the
  // point physics with zero values and gradients, so a pair term of an absent
  // grain is exactly zero; a warp skips the pair when no lane needs it.  The
  // full operator passes m = ~0u, which folds every test away.
  __device__ __forceinline__ bool pair_needed(unsigned m, int i, int j)
  {
    if (m == ~0u)
      return true;
    return __any_sync(0xffffffffu, ((m >> i) & (m >> j) & 1u) != 0u);
  }

  template <typename R>
  __device__ __forceinline__ R phi_clamped(R c)
  {
    return clamp01(c * c * c * (R(10) - R(15) * c + R(6) * c * c));
  }

  // ---------------------------------------------------------------------
  // Residual flux of the c row: M(c, eta, grad c, grad eta) grad mu
  // scalar: mobility.h:439-472, tensorial: mobility.h:756-804
  template <int DIM, int G, bool TENS, typename R>
  __device__ __forceinline__ void apply_M(const PhysR<R> &p, R c, const R (&eta)[gdim(G)], const R (&gc)[DIM],
                                          const R (*geta)[DIM], const R (&gmu)[DIM], R (&out)[DIM],
                                          unsigned m = ~0u)
  {
    const R phi = phi_clamped(c);
    if constexpr (!TENS)
      {
        R etaij = R(0);
#pragma unroll
        for (int i = 0; i < G; ++i)
#pragma unroll
          for (int j = 0; j < i; ++j)
            etaij += eta[i] * eta[j];
        const R M = p.Mvol * phi + p.Mvap * (R(1) - phi) + p.Msurf * R(4) * c * c * (R(1) - c) * (R(1) - c) +
                    (R(2) * p.Mgb) * etaij;
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          out[d] = M * gmu[d];
      }
    else
      {
        const R fvv   = p.Mvol * phi + p.Mvap * (R(1) - phi);
        const R fsurf = p.Msurf * R(4) * (c * c) * ((R(1) - c) * (R(1) - c));
        R       nc[DIM], n2, rs;
        unit_vector<DIM>(gc, nc, n2, rs);
        const R a  = fvv + fsurf * R(1.001);
        const R b  = fsurf * dotv<DIM>(nc, gmu);
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          out[d] = a * gmu[d] - nc[d] * b;
        if constexpr (G > 1)
          {
            // sum_{i>j} eta_i eta_j (grad mu - f_ij d_ij (d_ij . grad mu))
            R s1 = R(0), acc[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d)
              acc[d] = R(0);
#pragma unroll
            for (int i = 0; i < G; ++i)
#pragma unroll
              for (int j = 0; j < i; ++j)
                {
                  if (!pair_needed(m, i, j))
                    continue;
                  R dd[DIM];
#pragma unroll
                  for (int d = 0; d < DIM; ++d)
                    dd[d] = geta[i][d] - geta[j][d];
                  const R f  = unit_vector_filter_2<DIM>(dd);
                  const R pe = eta[i] * eta[j];
                  s1 += pe;
                  const R t = pe * f * dotv<DIM>(dd, gmu);
#pragma unroll
                  for (int d = 0; d < DIM; ++d)
                    acc[d] -= t * dd[d];
                }
            const R m2 = R(2) * p.Mgb;
#pragma unroll
            for (int d = 0; d < DIM; ++d)
              out[d] += m2 * (s1 * gmu[d] + acc[d]);
          }
      }
  }

  // ---------------------------------------------------------------------
  // Jacobian flux of the c row: d/du [M grad mu] applied to (dc, grad dc,
  // grad dmu, deta).  scalar: mobility.h:476-534, tensorial: mobility.h:808-916
  template <int DIM, int G, bool TENS, typename R>
  __device__ __forceinline__ void apply_M_derivative(const PhysR<R> &p, R c, const R (&gc)[DIM],
                                                     const R (&gmu)[DIM], const R (&eta)[gdim(G)], const R (*geta)[DIM],
                                                     R dc, const R (&gdc)[DIM], const R (&gdmu)[DIM],
                                                     const R (&deta)[gdim(G)], R (&out)[DIM], unsigned m = ~0u)
  {
    const R phi = phi_clamped(c);
    const R omc = R(1) - c;
    if constexpr (!TENS)
      {
        R eta_sum = R(0), eta_ij = R(0);
#pragma unroll
        for (int i = 0; i < G; ++i)
          {
            eta_sum += eta[i];
#pragma unroll
            for (int j = 0; j < i; ++j)
              eta_ij += eta[i] * eta[j];
          }
        const R M = p.Mvol * phi + p.Mvap * (R(1) - phi) + p.Msurf * R(4) * c * c * omc * omc + (R(2) * p.Mgb) * eta_ij;
        const R dphidc = R(30) * c * c * omc * omc;
        const R dMdc   = p.Mvol * dphidc - p.Mvap * dphidc + p.Msurf * R(8) * c * (R(1) - R(3) * c + R(2) * c * c);
        R       factor = R(0);
#pragma unroll
        for (int i = 0; i < G; ++i)
          factor += (eta_sum - eta[i]) * deta[i];
        const R k = dMdc * dc + (R(2) * p.Mgb) * factor;
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          out[d] = M * gdmu[d] + k * gmu[d];
      }
    else
      {
        R nc[DIM], n2, rs;
        unit_vector<DIM>(gc, nc, n2, rs);
        const R c2 = R(4) * c * c * omc * omc; // 4 c^2 (1-c)^2
        // 1) M
        const R fvv   = p.Mvol * phi + p.Mvap * (R(1) - phi);
        const R fsurf = p.Msurf * c2;
        const R nc_gdmu = dotv<DIM>(nc, gdmu);
        const R nc_gmu  = dotv<DIM>(nc, gmu);
        // 2) dM/dc (hpsint uses dphidc = 30 * 4 c^2 (1-c)^2 here, mobility.h:852-854)
        const R fvv2  = (p.Mvol - p.Mvap) * (R(30) * c2);
        R       dfs   = p.Msurf * R(8) * c * omc * (R(1) - R(2) * c);
        dfs           = sel(fsurf < R(1e-6), R(0), dfs);
        // 3) dM/dgrad c; |grad c| < 1e-4 (|grad c|^2 < 1e-8) counts as 1
        const R fs3   = sel(fsurf < R(1e-6), R(0), fsurf);
        const R inrm3 = sel(n2 < R(1e-8), R(1), rs);
        const R nc_gdc = dotv<DIM>(nc, gdc);
        R       temp[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          temp[d] = gdc[d] - nc[d] * nc_gdc;
        const R gmu_temp = dotv<DIM>(gmu, temp);
        const R k3       = -fs3 * inrm3;
        const R a2       = (fvv2 + dfs * R(1.001)) * dc;
        const R b2       = dfs * nc_gmu * dc;
        // (fvv + fsurf) grad dmu - nc (fsurf nc.grad dmu) + a2 grad mu - nc b2
        //   + k3 (nc.grad mu temp + nc grad mu.temp), the nc terms collected
        const R al = fvv + fsurf, be = fsurf * nc_gdmu + b2 - k3 * gmu_temp, ga = k3 * nc_gmu;
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          out[d] = al * gdmu[d] + a2 * gmu[d] - nc[d] * be + ga * temp[d];
        if constexpr (G > 1)
          {
            // 4) sum_{i>j} [ eta_i eta_j P_ij grad dmu + (eta_j deta_i + eta_i deta_j) P_ij grad mu ]
            //    with P_ij = I - f_ij d_ij d_ij^T, d_ij = grad eta_i - grad eta_j
            R s1 = R(0), s2 = R(0), acc[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d)
              acc[d] = R(0);
            // with many grains, d_ij . v = grad eta_i . v - grad eta_j . v from per-grain dots
            constexpr bool PER_GRAIN = G >= 5;
            R              ag[PER_GRAIN ? G : 1], bg[PER_GRAIN ? G : 1];
            if constexpr (PER_GRAIN)
              {
#pragma unroll
                for (int i = 0; i < G; ++i)
                  {
                    ag[i] = dotv<DIM>(geta[i], gdmu);
                    bg[i] = dotv<DIM>(geta[i], gmu);
                  }
              }
#pragma unroll
            for (int i = 0; i < G; ++i)
#pragma unroll
              for (int j = 0; j < i; ++j)
                {
                  if (!pair_needed(m, i, j))
                    continue;
                  R dd[DIM];
#pragma unroll
                  for (int d = 0; d < DIM; ++d)
                    dd[d] = geta[i][d] - geta[j][d];
                  const R f  = unit_vector_filter_2<DIM>(dd);
                  const R p1 = eta[i] * eta[j];
                  const R p2 = eta[j] * deta[i] + eta[i] * deta[j];
                  s1 += p1;
                  s2 += p2;
                  R da, db;
                  if constexpr (PER_GRAIN)
                    {
                      da = ag[i] - ag[j];
                      db = bg[i] - bg[j];
                    }
                  else
                    {
                      da = dotv<DIM>(dd, gdmu);
                      db = dotv<DIM>(dd, gmu);
                    }
                  const R t = f * (p1 * da + p2 * db);
#pragma unroll
                  for (int d = 0; d < DIM; ++d)
                    acc[d] -= t * dd[d];
                }
            const R m2 = R(2) * p.Mgb;
#pragma unroll
            for (int d = 0; d < DIM; ++d)
              out[d] += m2 * (s1 * gdmu[d] + s2 * gmu[d] + acc[d]);
          }
      }
  }

  // The mobility as a DIM x DIM matrix, M grad mu = apply_M(grad mu) for
  // every grad mu (mobility.h:439-472 scalar, :756-804 tensorial): one pass
  // over the grain pairs instead of one apply_M per unit vector.
  template <int DIM, int G, bool TENS, typename R>
  __device__ __forceinline__ void mobility_matrix(const PhysR<R> &p, R c, const R (&eta)[gdim(G)],
                                                  const R (&gc)[DIM], const R (*geta)[DIM], R (&Mm)[DIM][DIM])
  {
    const R phi = phi_clamped(c);
    if constexpr (!TENS)
      {
        R etaij = R(0);
#pragma unroll
        for (int i = 0; i < G; ++i)
#pragma unroll
          for (int j = 0; j < i; ++j)
            etaij += eta[i] * eta[j];
        const R M = p.Mvol * phi + p.Mvap * (R(1) - phi) + p.Msurf * R(4) * c * c * (R(1) - c) * (R(1) - c) +
                    (R(2) * p.Mgb) * etaij;
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int b = 0; b < DIM; ++b)
            Mm[a][b] = a == b ? M : R(0);
      }
    else
      {
        const R fvv   = p.Mvol * phi + p.Mvap * (R(1) - phi);
        const R fsurf = p.Msurf * R(4) * (c * c) * ((R(1) - c) * (R(1) - c));
        R       nc[DIM], n2, rs;
        unit_vector<DIM>(gc, nc, n2, rs);
        const R diag = fvv + fsurf * R(1.001);
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int b = 0; b < DIM; ++b)
            Mm[a][b] = (a == b ? diag : R(0)) - fsurf * nc[a] * nc[b];
        if constexpr (G > 1)
          {
            const R m2 = R(2) * p.Mgb;
            R       s1 = R(0), acc[DIM][DIM];
#pragma unroll
            for (int a = 0; a < DIM; ++a)
#pragma unroll
              for (int b = 0; b < DIM; ++b)
                acc[a][b] = R(0);
#pragma unroll 1
            for (int i = 0; i < G; ++i)
#pragma unroll 1
              for (int j = 0; j < i; ++j)
                {
                  R dd[DIM];
#pragma unroll
                  for (int d = 0; d < DIM; ++d)
                    dd[d] = geta[i][d] - geta[j][d];
                  const R f  = unit_vector_filter_2<DIM>(dd);
                  const R pe = eta[i] * eta[j];
                  s1 += pe;
                  const R t = pe * f;
#pragma unroll
                  for (int a = 0; a < DIM; ++a)
#pragma unroll
                    for (int b = 0; b < DIM; ++b)
                      acc[a][b] -= t * dd[a] * dd[b];
                }
#pragma unroll
            for (int a = 0; a < DIM; ++a)
#pragma unroll
              for (int b = 0; b < DIM; ++b)
                Mm[a][b] += m2 * ((a == b ? s1 : R(0)) + acc[a][b]);
          }
      }
  }

  // ---------------------------------------------------------------------
  // dM/dc applied to grad mu (a vector): scalar mobility.h:378-394,
  // tensorial mobility.h:668-696.  Used by the Cahn-Hilliard block tangent.
  template <int DIM, bool TENS, typename R>
  __device__ __forceinline__ void dM_dc_times(const PhysR<R> &p, R c, const R (&gc)[DIM], const R (&v)[DIM],
                                              R (&out)[DIM])
  {
    const R omc = R(1) - c;
    if constexpr (!TENS)
      {
        const R dphidc = R(30) * c * c * omc * omc;
        const R dMdc   = p.Mvol * dphidc - p.Mvap * dphidc + p.Msurf * R(8) * c * (R(1) - R(3) * c + R(2) * c * c);
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          out[d] = dMdc * v[d];
      }
    else
      {
        const R c2     = R(4) * c * c * omc * omc;
        const R dphidc = R(30) * c2;
        const R fsurf  = p.Msurf * c2;
        R       dfs    = p.Msurf * R(8) * c * omc * (R(1) - R(2) * c);
        dfs            = fsurf < R(1e-6) ? R(0) : dfs;
        R nc[DIM], n2, rs;
        unit_vector<DIM>(gc, nc, n2, rs);
        const R ncv = dotv<DIM>(nc, v);
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          out[d] = (p.Mvol - p.Mvap) * dphidc * v[d] + dfs * (R(1.001) * v[d] - nc[d] * ncv);
      }
  }

  // dM/d(grad c) as a DIM x DIM matrix K (row-major): tensorial
  // mobility.h:700-721, zero for scalar mobility (mobility.h:399-409).
  template <int DIM, bool TENS, typename R>
  __device__ __forceinline__ void dM_dgrad_c(const PhysR<R> &p, R c, const R (&gc)[DIM], const R (&gmu)[DIM],
                                             R (&K)[DIM][DIM])
  {
    if constexpr (!TENS)
      {
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int b = 0; b < DIM; ++b)
            K[a][b] = R(0);
      }
    else
      {
        R fsurf = p.Msurf * R(4) * (c * c) * ((R(1) - c) * (R(1) - c));
        R nc[DIM], n2, rs;
        unit_vector<DIM>(gc, nc, n2, rs);
        fsurf         = fsurf < R(1e-6) ? R(0) : fsurf;
        const R inrm3 = n2 < R(1e-8) ? R(1) : rs;
        const R ncmu  = dotv<DIM>(nc, gmu);
        // T = -fsurf (ncmu I + nc mu^T),  M = (I - nc nc^T) / nrm,  K = T M
        R Tm[DIM][DIM], Mm[DIM][DIM];
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int b = 0; b < DIM; ++b)
            {
              Tm[a][b] = -fsurf * ((a == b ? ncmu : R(0)) + nc[a] * gmu[b]);
              Mm[a][b] = ((a == b ? R(1) : R(0)) - nc[a] * nc[b]) * inrm3;
            }
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int b = 0; b < DIM; ++b)
            {
              R s = R(0);
#pragma unroll
              for (int e = 0; e < DIM; ++e)
                s += Tm[a][e] * Mm[e][b];
              K[a][b] = s;
            }
      }
  }
} // namespace sint
