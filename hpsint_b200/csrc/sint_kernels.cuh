// Cell kernels of the sintering operator (templates; instantiated per
// dimension, number of grains and mobility type in sint_inst_*.cu).
#pragma once

#include "sint_common.cuh"
#include "sint_physics.cuh"

namespace sint
{
  // Park a lane's node contribution in shared memory (zero for cells outside the mesh).
  template <int DIM, typename R>
  __device__ __forceinline__ void store_contrib(R *s_con, int comp, R r, bool valid)
  {
    using T = Tile<DIM>;
    s_con[comp * T::CS + (threadIdx.x & (T::NQ - 1)) * T::CP + threadIdx.x / T::NQ] = valid ? r : R(0);
  }

  // -------------------------------------------------------------------------
  // Jacobian-vector product: dst = J(lin) src.
  // SinteringOperatorGenericQuad::operator() (operator_sintering_generic.h:101-190)
  // inside do_vmult_range (:539-577).  The linearisation point is evaluated
  // from the nodal state instead of a quadrature-point cache.
  //
  // Only the c row has a point-dependent gradient flux (the mobility term); the
  // mu and eta rows have constant-coefficient gradient terms (-kappa_c grad dc,
  // L kappa_p grad deta), which are applied with the exact element stiffness
  // stencil to the nodal values, so those rows only integrate point values.
  //
  // Persistent and software pipelined: block b handles tiles b, b + grid, ...;
  // the node boxes of the next tile are copied (cp.async) into the second half
  // of a double buffer while the current tile is computed.
  template <int DIM, int G, bool TENS, typename R>
  __device__ __forceinline__ void jvp_tile(const Grid &g, const PhysR<R> &p, const R *s_lin, const R *s_src,
                                           R *s_con, const TileCoord &tc)
  {
    using T           = Tile<DIM>;
    const QP<DIM, R> w(g);
    const int        cell  = threadIdx.x / T::NQ;
    const int        b0    = cell_box_base<DIM>(cell);
    const bool       valid = cell_in_mesh<DIM>(cell, tc, g);

    // linearisation point at this quadrature point
    R c, gc[DIM], mu_unused, gmu[DIM];
    if constexpr (TENS)
      eval_vg<DIM>(s_lin, b0, w, c, gc);
    else
      c = eval_v<DIM>(s_lin, b0, w);
    eval_vg<DIM>(s_lin + T::BOX, b0, w, mu_unused, gmu);
    R eta[G];
    R geta[TENS ? G : 1][DIM];
#pragma unroll
    for (int i = 0; i < G; ++i)
      {
        if constexpr (TENS)
          eval_vg<DIM>(s_lin + (2 + i) * T::BOX, b0, w, eta[i], geta[i]);
        else
          eta[i] = eval_v<DIM>(s_lin + (2 + i) * T::BOX, b0, w);
      }
    // direction
    R dc, gdc[DIM], dmu, gdmu[DIM];
    if constexpr (TENS)
      eval_vg<DIM>(s_src, b0, w, dc, gdc);
    else
      dc = eval_v<DIM>(s_src, b0, w);
    eval_vg<DIM>(s_src + T::BOX, b0, w, dmu, gdmu);
    R deta[G];
#pragma unroll
    for (int i = 0; i < G; ++i)
      deta[i] = eval_v<DIM>(s_src + (2 + i) * T::BOX, b0, w);

    // free energy second derivatives at the linearisation point (free_energy.h:143-161)
    R s2 = R(0);
#pragma unroll
    for (int i = 0; i < G; ++i)
      s2 += eta[i] * eta[i];
    const R omc = R(1) - c;
    const R fcc = R(2) * p.A * (c * c) + R(4) * p.A * c * (R(2) * c - R(2)) + R(2) * p.A * (omc * omc) + R(2) * p.B;
    const R B12 = p.B * R(12);

    // 1) c row (generic.h:120-134)
    {
      R gres[DIM];
      apply_M_derivative<DIM, G, TENS>(p, c, gc, gmu, eta, geta, dc, gdc, gdmu, deta, gres);
      store_contrib<DIM>(s_con, 0, integrate_butterfly<DIM>(dc * p.w0, gres, w), valid);
    }
    // 2) mu row (generic.h:138-146): value part + (-kappa_c) K dc
    {
      R v = p.walg * dmu - fcc * dc;
#pragma unroll
      for (int i = 0; i < G; ++i)
        v -= B12 * eta[i] * (eta[i] - R(1)) * deta[i];
      const R r = integrate_value_butterfly<DIM>(v, w) - p.kc * stiffness_apply<DIM>(s_src, b0, w, g);
      store_contrib<DIM>(s_con, 1, r, valid);
    }
    // 3) eta rows (generic.h:150-163, free_energy.h:233-252): value part + L kappa_p K deta_i
    {
      R S = R(0);
#pragma unroll
      for (int i = 0; i < G; ++i)
        S += eta[i] * deta[i];
      const R cL24B = p.L * R(24) * p.B;
      const R Lkp   = p.L * p.kp;
#pragma unroll
      for (int i = 0; i < G; ++i)
        {
          const R e   = eta[i];
          const R fce = B12 * e * (e - R(1));
          const R fee = p.B * (R(12) - R(12) * c + R(2) * e * (R(12) * c - R(24)) + R(24) * (e * e) + R(12) * s2);
          R       v   = deta[i] * p.w0 + p.L * (fce * dc + fee * deta[i]);
          if constexpr (G > 1)
            v += cL24B * e * (S - e * deta[i]);
          const R r = integrate_value_butterfly<DIM>(v, w) +
                      Lkp * stiffness_apply<DIM>(s_src + (2 + i) * T::BOX, b0, w, g);
          store_contrib<DIM>(s_con, 2 + i, r, valid);
        }
    }
  }

  // Two resident blocks per SM (<= 128 registers) unless the FP64 grain state
  // of large G would spill; those run one block with up to 255 registers.
  template <int DIM, int G, bool TENS, typename R>
  __global__ void __launch_bounds__(Tile<DIM>::THREADS, (sizeof(R) == 8 && G > 5) ? 1 : 2)
    jvp_kernel(const Grid g, const Phys ph, const R *__restrict__ lin, const R *__restrict__ src,
               R *__restrict__ dst, R *__restrict__ partial)
  {
    using T          = Tile<DIM>;
    constexpr int C  = G + 2;
    constexpr int VB = 2 * C * T::BOX; // one buffer: linearisation point + direction
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *s_buf = reinterpret_cast<R *>(smem_raw); // 2 x VB
    R *s_con = s_buf + 2 * VB;

    const PhysR<R> p(ph);
    long long      tile = blockIdx.x;
    if (tile < g.n_tiles)
      {
        const BoxNode<DIM> bn(g, tile_coord_of<DIM>(g, tile));
        load_box_async<DIM>(s_buf, lin, C, g, bn);
        load_box_async<DIM>(s_buf + C * T::BOX, src, C, g, bn);
      }
    cp_async_commit();
    for (int it = 0; tile < g.n_tiles; ++it, tile += gridDim.x)
      {
        const long long next = tile + gridDim.x;
        R              *nb   = s_buf + ((it + 1) & 1) * VB;
        if (next < g.n_tiles)
          {
            const BoxNode<DIM> bnn(g, tile_coord_of<DIM>(g, next));
            load_box_async<DIM>(nb, lin, C, g, bnn);
            load_box_async<DIM>(nb + C * T::BOX, src, C, g, bnn);
          }
        cp_async_commit();
        cp_async_wait<1>(); // this tile's group has landed (only the prefetch may be pending)
        __syncthreads();
        const TileCoord tc = tile_coord_of<DIM>(g, tile);
        const R        *cb = s_buf + (it & 1) * VB;
        jvp_tile<DIM, G, TENS, R>(g, p, cb, cb + C * T::BOX, s_con, tc);
        __syncthreads();
        sum_and_store<DIM>(s_con, C, g, tc, BoxNode<DIM>(g, tc), dst, partial);
        __syncthreads(); // s_con and this buffer are reused by the next iterations
      }
    cp_async_wait<0>();
  }

  // -------------------------------------------------------------------------
  // Nonlinear residual: dst = R(src), SinteringOperatorGenericResidualQuad
  // (operator_sintering_generic.h:254-308) with the history of
  // do_evalute_history (:927-975) for WTD == 2.  As in the Jacobian, the mu and
  // eta rows' constant-coefficient gradient terms use the stiffness stencil.
  template <int DIM, int G, bool TENS, int WTD>
  __global__ void __launch_bounds__(Tile<DIM>::THREADS)
    residual_kernel(const Grid g, const Phys ph, const double *__restrict__ src, const double *__restrict__ h0,
                    const double *__restrict__ h1, const double *__restrict__ h2, double *__restrict__ dst,
                    double *__restrict__ partial)
  {
    using R          = double;
    using T          = Tile<DIM>;
    constexpr int C  = G + 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *s_u   = reinterpret_cast<R *>(smem_raw);
    R *s_h   = s_u + C * T::BOX;
    R *s_con = s_h + (WTD == 2 ? C : 0) * T::BOX;

    const TileCoord    tc = tile_coord<DIM>(g);
    const BoxNode<DIM> bn(g, tc);
    load_box<DIM>(s_u, src, C, g, bn);
    if constexpr (WTD == 2)
      {
        // sum_i w_{i+1} u_old_i at the nodes (generic.h:947-966); mu has no history
        if (bn.active)
          for (int comp = bn.grp; comp < C; comp += T::NG)
            {
              R v = R(0);
              if (comp != 1 && bn.inside)
                {
                  const long long off = comp * g.ld + bn.gidx;
                  v                   = h0[off] * ph.w_hist[0];
                  if (ph.order > 1)
                    v += h1[off] * ph.w_hist[1];
                  if (ph.order > 2)
                    v += h2[off] * ph.w_hist[2];
                }
              s_h[comp * T::BOX + bn.b] = v;
            }
      }
    __syncthreads();

    const PhysR<R>   p(ph);
    const QP<DIM, R> w(g);
    const int        cell  = threadIdx.x / T::NQ;
    const int        b0    = cell_box_base<DIM>(cell);
    const bool       valid = cell_in_mesh<DIM>(cell, tc, g);

    R c, gc[DIM], mu, gmu[DIM];
    if constexpr (TENS)
      eval_vg<DIM>(s_u, b0, w, c, gc);
    else
      c = eval_v<DIM>(s_u, b0, w);
    eval_vg<DIM>(s_u + T::BOX, b0, w, mu, gmu);
    R eta[G];
    R geta[TENS ? G : 1][DIM];
#pragma unroll
    for (int i = 0; i < G; ++i)
      {
        if constexpr (TENS)
          eval_vg<DIM>(s_u + (2 + i) * T::BOX, b0, w, eta[i], geta[i]);
        else
          eta[i] = eval_v<DIM>(s_u + (2 + i) * T::BOX, b0, w);
      }

    R s2 = R(0), s3 = R(0);
#pragma unroll
    for (int i = 0; i < G; ++i)
      {
        s2 += eta[i] * eta[i];
        s3 += eta[i] * eta[i] * eta[i];
      }
    const R omc = R(1) - c;

    // 1) c row (generic.h:275-285)
    {
      R v = R(0);
      if constexpr (WTD >= 1)
        v = c * p.w0;
      if constexpr (WTD == 2)
        v += eval_v<DIM>(s_h, b0, w);
      R gres[DIM];
      apply_M<DIM, G, TENS>(p, c, eta, gc, geta, gmu, gres);
      store_contrib<DIM>(s_con, 0, integrate_butterfly<DIM>(v, gres, w), valid);
    }
    // 2) mu row (generic.h:288-289, free_energy.h:124-134): value part - kappa_c K c
    {
      const R df_dc = p.A * (c * c) * (R(2) * c - R(2)) + R(2) * p.A * c * (omc * omc) +
                      p.B * (R(2) * c - R(6) * s2 + R(4) * s3);
      const R r = integrate_value_butterfly<DIM>(p.walg * mu - df_dc, w) - p.kc * stiffness_apply<DIM>(s_u, b0, w, g);
      store_contrib<DIM>(s_con, 1, r, valid);
    }
    // 3) eta rows (generic.h:293-304, free_energy.h:136-141): value part + L kappa_p K eta_i
    {
      const R Lkp = p.L * p.kp;
#pragma unroll
      for (int i = 0; i < G; ++i)
        {
          const R e = eta[i];
          R       v = p.L * (e * (p.B * R(12)) * (e * (c - R(2)) + omc + s2));
          if constexpr (WTD >= 1)
            v += e * p.w0;
          if constexpr (WTD == 2)
            v += eval_v<DIM>(s_h + (2 + i) * T::BOX, b0, w);
          const R r = integrate_value_butterfly<DIM>(v, w) +
                      Lkp * stiffness_apply<DIM>(s_u + (2 + i) * T::BOX, b0, w, g);
          store_contrib<DIM>(s_con, 2 + i, r, valid);
        }
    }
    __syncthreads();
    sum_and_store<DIM>(s_con, C, g, tc, bn, dst, partial);
  }

  // -------------------------------------------------------------------------
  // Preconditioner diagonals at the linearisation point (FP64), G + 4 outputs:
  //   [0..3] node-diagonal 2x2 block of the Cahn-Hilliard tangent
  //          (OperatorCahnHilliard, sintering/preconditioners.h:110-168):
  //          J_cc, J_c,mu, J_mu,c, J_mu,mu
  //   [4..]  diagonal of OperatorAllenCahn (preconditioners.h:364-394)
  // Each thread first computes its point's coefficients (mobility matrix M,
  // dM/dc grad mu, dM/dgrad c, f_cc, f_eta_i eta_i), then, as the owner of
  // local node l, sums phi_l / grad phi_l weighted terms over the cell's points.
  template <int DIM, int G, bool TENS>
  struct DiagLayout
  {
    static constexpr int NOUT  = G + 4;
    static constexpr int NCOEF = DIM * DIM + DIM + DIM * DIM + 1 + G;
  };

  template <int DIM, int G, bool TENS>
  __global__ void __launch_bounds__(Tile<DIM>::THREADS)
    diag_kernel(const Grid g, const Phys ph, const double *__restrict__ lin, double *__restrict__ dst,
                double *__restrict__ partial)
  {
    using R          = double;
    using T          = Tile<DIM>;
    using LY         = DiagLayout<DIM, G, TENS>;
    constexpr int C  = G + 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *s_lin  = reinterpret_cast<R *>(smem_raw);
    R *s_coef = s_lin + C * T::BOX;
    R *s_con  = s_coef + LY::NCOEF * T::THREADS; // NOUT * CS

    const TileCoord    tc = tile_coord<DIM>(g);
    const BoxNode<DIM> bn(g, tc);
    load_box<DIM>(s_lin, lin, C, g, bn);
    __syncthreads();

    const PhysR<R>   p(ph);
    const QP<DIM, R> w(g);
    const int        cell  = threadIdx.x / T::NQ;
    const int        b0    = cell_box_base<DIM>(cell);
    const bool       valid = cell_in_mesh<DIM>(cell, tc, g);

    {
      R c, gc[DIM], mu_unused, gmu[DIM];
      eval_vg<DIM>(s_lin, b0, w, c, gc);
      eval_vg<DIM>(s_lin + T::BOX, b0, w, mu_unused, gmu);
      R eta[G];
      R geta[G][DIM];
#pragma unroll
      for (int i = 0; i < G; ++i)
        eval_vg<DIM>(s_lin + (2 + i) * T::BOX, b0, w, eta[i], geta[i]);
      R *cf = s_coef + threadIdx.x * LY::NCOEF;
      // mobility matrix: column e = apply_M(..., unit vector e)
#pragma unroll
      for (int e = 0; e < DIM; ++e)
        {
          R unit[DIM], col[DIM];
#pragma unroll
          for (int d = 0; d < DIM; ++d)
            unit[d] = d == e ? R(1) : R(0);
          apply_M<DIM, G, TENS>(p, c, eta, gc, geta, unit, col);
#pragma unroll
          for (int d = 0; d < DIM; ++d)
            cf[d * DIM + e] = col[d];
        }
      R m[DIM];
      dM_dc_times<DIM, TENS>(p, c, gc, gmu, m);
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        cf[DIM * DIM + d] = m[d];
      R K[DIM][DIM];
      dM_dgrad_c<DIM, TENS>(p, c, gc, gmu, K);
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b)
          cf[DIM * DIM + DIM + a * DIM + b] = K[a][b];
      const R omc = R(1) - c;
      R       s2  = R(0);
#pragma unroll
      for (int i = 0; i < G; ++i)
        s2 += eta[i] * eta[i];
      cf[2 * DIM * DIM + DIM] =
        R(2) * p.A * (c * c) + R(4) * p.A * c * (R(2) * c - R(2)) + R(2) * p.A * (omc * omc) + R(2) * p.B;
#pragma unroll
      for (int i = 0; i < G; ++i)
        {
          const R e = eta[i];
          cf[2 * DIM * DIM + DIM + 1 + i] =
            p.B * (R(12) - R(12) * c + R(2) * e * (R(12) * c - R(24)) + R(24) * (e * e) + R(12) * s2);
        }
    }
    __syncthreads();

    {
      // this thread is the owner of local node l = lane bits
      const int l = threadIdx.x & (T::NQ - 1);
      R         acc[LY::NOUT];
#pragma unroll
      for (int k = 0; k < LY::NOUT; ++k)
        acc[k] = R(0);
      for (int q = 0; q < T::NQ; ++q)
        {
          const R *cf = s_coef + (cell * T::NQ + q) * LY::NCOEF;
          // phi_l(x_q) and grad phi_l(x_q)
          R phi = R(1), dphi[DIM];
#pragma unroll
          for (int d = 0; d < DIM; ++d)
            {
              const int ld = (l >> d) & 1, qd = (q >> d) & 1;
              phi *= (ld == qd) ? w.g1 : w.g0;
            }
#pragma unroll
          for (int d = 0; d < DIM; ++d)
            {
              R v = (((l >> d) & 1) ? R(1) : R(-1)) * w.ih[d];
#pragma unroll
              for (int e = 0; e < DIM; ++e)
                if (e != d)
                  v *= (((l >> e) & 1) == ((q >> e) & 1)) ? w.g1 : w.g0;
              dphi[d] = v;
            }
          const R *Mm = cf;
          const R *mv = cf + DIM * DIM;
          const R *Km = cf + DIM * DIM + DIM;
          const R  fcc = cf[2 * DIM * DIM + DIM];
          R        gg = R(0), MphiPhi = R(0), KphiPhi = R(0), mphi = R(0);
#pragma unroll
          for (int a = 0; a < DIM; ++a)
            {
              gg += dphi[a] * dphi[a];
              mphi += mv[a] * dphi[a];
#pragma unroll
              for (int b = 0; b < DIM; ++b)
                {
                  MphiPhi += dphi[a] * Mm[a * DIM + b] * dphi[b];
                  KphiPhi += dphi[a] * Km[a * DIM + b] * dphi[b];
                }
            }
          const R pp = phi * phi;
          acc[0] += w.JxW * (p.w0 * pp + phi * mphi + KphiPhi);
          acc[1] += w.JxW * MphiPhi;
          acc[2] += w.JxW * (-fcc * pp - p.kc * gg);
          acc[3] += w.JxW * (p.walg * pp);
#pragma unroll
          for (int i = 0; i < G; ++i)
            acc[4 + i] += w.JxW * ((p.w0 + p.L * cf[2 * DIM * DIM + DIM + 1 + i]) * pp + p.L * p.kp * gg);
        }
#pragma unroll
      for (int k = 0; k < LY::NOUT; ++k)
        store_contrib<DIM>(s_con, k, acc[k], valid);
    }
    __syncthreads();
    sum_and_store<DIM>(s_con, LY::NOUT, g, tc, bn, dst, partial);
  }
} // namespace sint
