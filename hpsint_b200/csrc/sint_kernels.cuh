// Cell kernels of the sintering operator (templates; instantiated per
// dimension, number of grains and mobility type in sint_inst_*.cu).
#pragma once

#include "sint_cellfact.cuh"
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
  // Three-phase cell kernels (Jacobian-vector product and residual).
  //
  // Per tile: phase 1 evaluates every needed component at all points of a cell
  // (one thread per (cell, component), per-cell sum factorisation) into the
  // point-field buffer F[slot][cell]; phase 2 runs the point physics (one
  // thread per (point, cell)) and writes the point results to P[res][q][cell];
  // phase 3 integrates each residual row of a cell (one thread per (cell,
  // row)) into the node contributions K[row][l][cell] (aliasing F); the node
  // sum and the tile-face partials follow.  Warps always work on 32
  // consecutive cells of one component/point/row, so the shared-memory
  // accesses of the three phases are free of bank conflicts.
  //
  // Only the c row has a point-dependent gradient flux (mobility); the mu and
  // eta rows' gradient terms (-kappa_c grad c, L kappa_p grad eta) have
  // constant coefficients and are applied with the exact element stiffness to
  // the nodal values, so those rows integrate point values only.

  // Components evaluated in phase 1, in slot order.  Jacobian product:
  //   tensorial: [lin c, lin mu, lin eta_i] (value + gradient),
  //              [src c, src mu] (value + gradient), [src eta_i] (value)
  //   scalar:    [lin mu, src mu] (value + gradient),
  //              [lin c, lin eta_i, src c, src eta_i] (value)
  // Residual (u = the state, h = the weighted history):
  //   tensorial: [c, mu, eta_i] (value + gradient), [h c, h eta_i] (value)
  //   scalar:    [mu] (value + gradient), [c, eta_i] (value), [h c, h eta_i] (value)
  template <int DIM, int G, bool TENS, bool JVP, bool HIST>
  struct FieldMap
  {
    using SL = Slots<DIM>;
    static constexpr int NVG    = JVP ? (TENS ? 4 + G : 2) : (TENS ? 2 + G : 1);
    static constexpr int NV     = JVP ? (TENS ? G : 2 + 2 * G) : ((TENS ? 0 : 1 + G) + (HIST ? 1 + G : 0));
    static constexpr int NITEMS = NVG + NV;
    static constexpr int NSLOT  = NVG * SL::VG + NV * SL::V;

    __host__ __device__ static constexpr int base(int item)
    {
      return item < NVG ? item * SL::VG : NVG * SL::VG + (item - NVG) * SL::V;
    }
    // item index of each quantity (residual: "lin" is the state itself)
    static constexpr int lin_c  = TENS ? 0 : (JVP ? 2 : 1);
    static constexpr int lin_mu = TENS ? 1 : 0;
    __host__ __device__ static constexpr int lin_eta(int i) { return TENS ? 2 + i : (JVP ? 3 + i : 2 + i); }
    static constexpr int src_c  = TENS ? 2 + G : 3 + G;
    static constexpr int src_mu = TENS ? 3 + G : 1;
    __host__ __device__ static constexpr int src_eta(int i) { return 4 + G + i; }
    static constexpr int h_c = 2 + G;
    __host__ __device__ static constexpr int h_eta(int i) { return 3 + G + i; }
    // grain of a phase-1 item (-1 for c and mu items)
    __host__ __device__ static constexpr int grain(int it)
    {
      return (it >= lin_eta(0) && it < lin_eta(0) + G) ? it - lin_eta(0)
             : (JVP && it >= src_eta(0)) ? it - src_eta(0)
             : (!JVP && HIST && it >= h_eta(0)) ? it - h_eta(0)
                                               : -1;
    }

    // phase 1 item -> (buffer 0 = lin / state, 1 = src / history; component; value+gradient?)
    __device__ static void source(int it, int &buf, int &comp)
    {
      if constexpr (JVP)
        {
          if constexpr (TENS)
            {
              if (it < 2 + G) { buf = 0; comp = it; }
              else if (it < 4 + G) { buf = 1; comp = it - 2 - G; }
              else { buf = 1; comp = 2 + (it - 4 - G); }
            }
          else
            {
              if (it == 0) { buf = 0; comp = 1; }
              else if (it == 1) { buf = 1; comp = 1; }
              else if (it == 2) { buf = 0; comp = 0; }
              else if (it < 3 + G) { buf = 0; comp = 2 + (it - 3); }
              else if (it == 3 + G) { buf = 1; comp = 0; }
              else { buf = 1; comp = 2 + (it - 4 - G); }
            }
        }
      else
        {
          if constexpr (TENS)
            {
              if (it < 2 + G) { buf = 0; comp = it; }
              else if (it == 2 + G) { buf = 1; comp = 0; }
              else { buf = 1; comp = 2 + (it - 3 - G); }
            }
          else
            {
              if (it == 0) { buf = 0; comp = 1; }
              else if (it == 1) { buf = 0; comp = 0; }
              else if (it < 2 + G) { buf = 0; comp = 2 + (it - 2); }
              else if (it == 2 + G) { buf = 1; comp = 0; }
              else { buf = 1; comp = 2 + (it - 3 - G); }
            }
        }
    }
  };

  // Phase 1: evaluate all items of the tile.  With the grain cut-off (CUT),
  // the items of a grain absent on this thread's cell (bit clear in m) are
  // zero; a warp that has no lane needing an item writes the zeros without
  // evaluating.
  template <int DIM, int G, bool TENS, bool JVP, bool HIST, typename R, bool CUT = false>
  __device__ __forceinline__ void phase_evaluate(const R *box0, const R *box1, R *F, const CellConsts<DIM, R> &k,
                                                 unsigned m = ~0u)
  {
    using T            = Tile<DIM>;
    using SL           = Slots<DIM>;
    using FM           = FieldMap<DIM, G, TENS, JVP, HIST>;
    constexpr int NGRP = T::THREADS / T::CELLS;
    const int     cell = threadIdx.x % T::CELLS;
    const int     b0   = cell_box_base<DIM>(cell);
    for (int it = threadIdx.x / T::CELLS; it < FM::NITEMS; it += NGRP)
      {
        bool absent = false;
        if constexpr (CUT)
          {
            const int gr = FM::grain(it);
            absent       = gr >= 0 && ((m >> gr) & 1u) == 0u;
            if (!__any_sync(0xffffffffu, !absent))
              {
                const int ns = it < FM::NVG ? SL::VG : SL::V;
                for (int sl = 0; sl < ns; ++sl)
                  F[(FM::base(it) + sl) * T::CELLS + cell] = R(0);
                continue;
              }
          }
        int buf = 0, comp = 0;
        FM::source(it, buf, comp);
        R u[1 << DIM];
        cell_nodes<DIM>((buf == 0 ? box0 : box1) + comp * T::BOXS, b0, u);
        if constexpr (CUT)
          if (absent)
#pragma unroll
            for (int l = 0; l < (1 << DIM); ++l)
              u[l] = R(0);
        if (it < FM::NVG)
          cell_eval_vg<DIM>(u, k, F, FM::base(it), cell);
        else
          cell_eval_v<DIM>(u, k, F, FM::base(it), cell);
      }
  }

  // point-field accessors for phase 2 (thread = (point q, cell))
  template <int DIM, typename R>
  __device__ __forceinline__ R fval(const R *F, int base, int q, int cell)
  {
    return F[(base + q) * Tile<DIM>::CELLS + cell];
  }
  template <int DIM, typename R>
  __device__ __forceinline__ void fgrad(const R *F, int base, int q, int cell, R (&g)[DIM])
  {
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      g[d] = F[(base + Slots<DIM>::NQ + d * Slots<DIM>::NG1 + grad_slot<DIM>(d, q)) * Tile<DIM>::CELLS + cell];
  }

  // point results: P[(res * NQ + q) * CELLS + cell]; res 0 = c row value,
  // 1..DIM = c row flux, DIM + 1 = mu row value, DIM + 2 + i = eta_i row value
  template <int DIM, typename R>
  __device__ __forceinline__ void pstore(R *P, int res, int q, int cell, nd<R> v)
  {
    P[(res * Slots<DIM>::NQ + q) * Tile<DIM>::CELLS + cell] = v;
  }

  // Phase 2 of the Jacobian product at point q of cell `cell`
  // (SinteringOperatorGenericQuad::operator(), generic.h:101-190).
  template <int DIM, int G, bool TENS, typename R>
  __device__ __forceinline__ void jvp_point(const PhysR<R> &p, const R *F, R *P, int q, int cell, unsigned m = ~0u)
  {
    using FM = FieldMap<DIM, G, TENS, true, false>;
    R c, gc[DIM], gmu[DIM];
    c = fval<DIM>(F, FM::base(FM::lin_c), q, cell);
    if constexpr (TENS)
      fgrad<DIM>(F, FM::base(FM::lin_c), q, cell, gc);
    fgrad<DIM>(F, FM::base(FM::lin_mu), q, cell, gmu);
    R eta[gdim(G)];
    R geta[TENS ? gdim(G) : 1][DIM];
#pragma unroll
    for (int i = 0; i < G; ++i)
      {
        eta[i] = fval<DIM>(F, FM::base(FM::lin_eta(i)), q, cell);
        if constexpr (TENS)
          fgrad<DIM>(F, FM::base(FM::lin_eta(i)), q, cell, geta[i]);
      }
    R dc, gdc[DIM], dmu, gdmu[DIM];
    dc = fval<DIM>(F, FM::base(FM::src_c), q, cell);
    if constexpr (TENS)
      fgrad<DIM>(F, FM::base(FM::src_c), q, cell, gdc);
    dmu = fval<DIM>(F, FM::base(FM::src_mu), q, cell);
    fgrad<DIM>(F, FM::base(FM::src_mu), q, cell, gdmu);
    R deta[gdim(G)];
#pragma unroll
    for (int i = 0; i < G; ++i)
      deta[i] = fval<DIM>(F, FM::base(FM::src_eta(i)), q, cell);

    // free energy second derivatives at the linearisation point (free_energy.h:143-161)
    R s2 = R(0);
#pragma unroll
    for (int i = 0; i < G; ++i)
      s2 += eta[i] * eta[i];
    const R omc = R(1) - c;
    const R fcc = R(2) * p.A * (c * c) + R(4) * p.A * c * (R(2) * c - R(2)) + R(2) * p.A * (omc * omc) + R(2) * p.B;
    const R B12 = p.B * R(12);
    // f_{c eta_i} = 12 B eta_i (eta_i - 1) (free_energy.h:150-152), shared by the mu
    // and eta rows; f_{eta_i eta_i} = B (12 - 12 c + 2 eta_i (12 c - 24) + 24 eta_i^2
    // + 12 sum eta^2) (:154-158) in Horner form: f0 + eta_i (f1 + f2 eta_i)
    R fce[gdim(G)];
#pragma unroll
    for (int i = 0; i < G; ++i)
      {
        const R be = B12 * eta[i];
        fce[i]     = be * eta[i] - be;
      }
    const R fee0 = B12 * ((R(1) - c) + s2), fee1 = p.B * (R(24) * c - R(48)), fee2 = p.B * R(24);

    // 1) c row (generic.h:120-134)
    {
      R gres[DIM];
      apply_M_derivative<DIM, G, TENS>(p, c, gc, gmu, eta, geta, dc, gdc, gdmu, deta, gres, m);
      pstore<DIM>(P, 0, q, cell, dc * p.w0);
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        pstore<DIM>(P, 1 + d, q, cell, gres[d]);
    }
    // 2) mu row value (generic.h:138-144)
    {
      R v = p.walg * dmu - fcc * dc;
#pragma unroll
      for (int i = 0; i < G; ++i)
        v -= fce[i] * deta[i];
      pstore<DIM>(P, DIM + 1, q, cell, v);
    }
    // 3) eta row values (generic.h:150-163, free_energy.h:233-252)
    {
      R S = R(0);
#pragma unroll
      for (int i = 0; i < G; ++i)
        S += eta[i] * deta[i];
      const R cL24B = p.L * R(24) * p.B;
#pragma unroll
      for (int i = 0; i < G; ++i)
        {
          const R e   = eta[i];
          const R fee = fee0 + e * (fee1 + fee2 * e);
          R       v   = deta[i] * p.w0 + p.L * (fce[i] * dc + fee * deta[i]);
          if constexpr (G > 1)
            v += (cL24B * e) * (S - e * deta[i]);
          pstore<DIM>(P, DIM + 2 + i, q, cell, v);
        }
    }
  }

  // Phase 2 of the residual at point q of cell `cell`
  // (SinteringOperatorGenericResidualQuad::operator(), generic.h:254-308).
  template <int DIM, int G, bool TENS, int WTD, typename R>
  __device__ __forceinline__ void residual_point(const PhysR<R> &p, const R *F, R *P, int q, int cell,
                                                 unsigned m = ~0u)
  {
    using FM = FieldMap<DIM, G, TENS, false, WTD == 2>;
    R c, gc[DIM], mu, gmu[DIM];
    c = fval<DIM>(F, FM::base(FM::lin_c), q, cell);
    if constexpr (TENS)
      fgrad<DIM>(F, FM::base(FM::lin_c), q, cell, gc);
    mu = fval<DIM>(F, FM::base(FM::lin_mu), q, cell);
    fgrad<DIM>(F, FM::base(FM::lin_mu), q, cell, gmu);
    R eta[gdim(G)];
    R geta[TENS ? gdim(G) : 1][DIM];
#pragma unroll
    for (int i = 0; i < G; ++i)
      {
        eta[i] = fval<DIM>(F, FM::base(FM::lin_eta(i)), q, cell);
        if constexpr (TENS)
          fgrad<DIM>(F, FM::base(FM::lin_eta(i)), q, cell, geta[i]);
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
        v += fval<DIM>(F, FM::base(FM::h_c), q, cell);
      R gres[DIM];
      apply_M<DIM, G, TENS>(p, c, eta, gc, geta, gmu, gres, m);
      pstore<DIM>(P, 0, q, cell, v);
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        pstore<DIM>(P, 1 + d, q, cell, gres[d]);
    }
    // 2) mu row value (generic.h:288, free_energy.h:124-134)
    {
      const R df_dc = p.A * (c * c) * (R(2) * c - R(2)) + R(2) * p.A * c * (omc * omc) +
                      p.B * (R(2) * c - R(6) * s2 + R(4) * s3);
      pstore<DIM>(P, DIM + 1, q, cell, p.walg * mu - df_dc);
    }
    // 3) eta row values (generic.h:293-302, free_energy.h:136-141)
#pragma unroll
    for (int i = 0; i < G; ++i)
      {
        const R e = eta[i];
        R       v = p.L * (e * (p.B * R(12)) * (e * (c - R(2)) + omc + s2));
        if constexpr (WTD >= 1)
          v += e * p.w0;
        if constexpr (WTD == 2)
          v += fval<DIM>(F, FM::base(FM::h_eta(i)), q, cell);
        pstore<DIM>(P, DIM + 2 + i, q, cell, v);
      }
  }

  // Global coordinates of local cell `cell` of tile tc; false outside the mesh.
  template <int DIM>
  __device__ __forceinline__ bool cell_global(int cell, const TileCoord &tc, const Grid &g, int (&cc)[3])
  {
    using T = Tile<DIM>;
    cc[0]   = tc.o[0] + cell % T::TX;
    cc[1]   = tc.o[1] + (cell / T::TX) % T::TY;
    cc[2]   = DIM == 3 ? tc.o[2] + cell / (T::TX * T::TY) : 0;
    return cc[0] < g.n[0] && cc[1] < g.n[1] && (DIM == 2 || cc[2] < g.n[2]);
  }

  // Advection coefficients of one tile, staged once per tile before phase 1
  // (AdvectionVelocityData::reinit, sintering/advection.h:185-222): for
  // grain k (the tile's k-th grain under the cut-off) and local cell `cell`,
  // item i = k * CELLS + cell: vel[6 i ..] = the velocity at the cell's lower
  // corner and the angular velocity, has[i] = 1 when the grain has a segment
  // on the cell.  The velocity at point q is then vel + w x (x_q - corner).
  template <int DIM, int G, typename R, bool CUT>
  __device__ __forceinline__ void adv_stage(const AdvData &a, const Grid &g, const TileCoord &tc,
                                            unsigned long long gl, R *vel, unsigned char *has)
  {
    using T                 = Tile<DIM>;
    const long long n_cells = (long long)g.n[0] * g.n[1] * g.n[2];
    for (int it = threadIdx.x; it < G * T::CELLS; it += T::THREADS)
      {
        const int k = it / T::CELLS, cell = it % T::CELLS;
        int       cc[3];
        int       s = -1;
        if (cell_global<DIM>(cell, tc, g, cc))
          {
            const int b = CUT ? int((gl >> (4 * k)) & 15ull) : k;
            s           = a.cell_segments[b * n_cells + cc[0] + (long long)g.n[0] * (cc[1] + (long long)g.n[1] * cc[2])];
            if (s >= a.n_segments)
              s = -1;
          }
        has[it] = s >= 0;
        if (s >= 0)
          {
            const double *d    = a.segments + 9 * (long long)s;
            double        r[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int e = 0; e < DIM; ++e)
              r[e] = a.origin[e] + cc[e] * g.h[e] - d[6 + e];
            R *o = vel + 6 * it;
            o[0] = R(d[0] + d[4] * r[2] - d[5] * r[1]);
            o[1] = R(d[1] + d[5] * r[0] - d[3] * r[2]);
            o[2] = R(d[2] + d[3] * r[1] - d[4] * r[0]);
            o[3] = R(d[3]);
            o[4] = R(d[4]);
            o[5] = R(d[5]);
          }
      }
  }

  // Velocity of staged item `it` at point q (offset dq from the cell corner).
  template <int DIM, typename R>
  __device__ __forceinline__ void adv_velocity(const R *vel, int it, const R (&dq)[3], R (&v)[DIM])
  {
    const R *w = vel + 6 * it;
    v[0]       = w[0] + (w[4] * dq[2] - w[5] * dq[1]);
    v[1]       = w[1] + (w[5] * dq[0] - w[3] * dq[2]);
    if constexpr (DIM == 3)
      v[2] = w[2] + (w[3] * dq[1] - w[4] * dq[0]);
  }

  template <int DIM, typename R>
  __device__ __forceinline__ void adv_offset(const CellConsts<DIM, R> &k, const Grid &g, int q, R (&dq)[3])
  {
#pragma unroll
    for (int e = 0; e < 3; ++e)
      dq[e] = e < DIM ? (((q >> e) & 1) ? k.x1 : k.x0) * R(g.h[e]) : R(0);
  }

  // Advection of the c row at point q (phase 2, after the point physics):
  // the c flux loses v_i c for every grain i with a velocity on the cell, one
  // grain after the other (operator_sintering_generic.h:1015-1036 for the
  // residual, :167-177 for J v, where c is the direction's value).  With the
  // grain cut-off only the cell's relevant grains move it (AdvectionVelocityData
  // maps order parameters through the relevant-grain table,
  // sintering/advection.h:225-245).
  template <int DIM, int G, typename R, bool CUT>
  __device__ __forceinline__ void advect_c_point(const CellConsts<DIM, R> &k, const Grid &g, const R *F, int c_base,
                                                 R *P, int q, int cell, unsigned m, const R *vel,
                                                 const unsigned char *has)
  {
    using T = Tile<DIM>;
    R     dq[3];
    adv_offset<DIM>(k, g, q, dq);
    const R c = fval<DIM>(F, c_base, q, cell);
    R       flux[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      flux[d] = P[((1 + d) * Slots<DIM>::NQ + q) * T::CELLS + cell];
#pragma unroll 1
    for (int i = 0; i < G; ++i)
      {
        if ((CUT && ((m >> i) & 1u) == 0u) || !has[i * T::CELLS + cell])
          continue;
        R v[DIM];
        adv_velocity<DIM>(vel, i * T::CELLS + cell, dq, v);
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          flux[d] = flux[d] - v[d] * c;
      }
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      P[((1 + d) * Slots<DIM>::NQ + q) * T::CELLS + cell] = flux[d];
  }

  // Phase 3, 3D: the c row's contributions to the local nodes with z bit HZ
  // (K rows l = lx + 2 ly + 4 HZ) from the point values and fluxes in P.
  template <int HZ, typename R>
  __device__ __forceinline__ void integrate_c_row_half(const R *P, const CellConsts<3, R> &k, int cell, bool in,
                                                       bool in_b, R *K)
  {
    using T          = Tile<3>;
    constexpr int NQ = 8;
    R v[NQ], gg[3][NQ], r[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q)
      {
        v[q] = P[(0 * NQ + q) * T::CELLS + cell];
#pragma unroll
        for (int d = 0; d < 3; ++d)
          gg[d][q] = P[((1 + d) * NQ + q) * T::CELLS + cell];
      }
    cell_integrate_vg_half<HZ>(v, gg, k, r);
#pragma unroll
    for (int l = 4 * HZ; l < 4 * HZ + 4; ++l)
      K[l * T::CP + cell] = (in && in_b) ? r[l] : lane_keep(r[l], in, in_b);
  }

  // Phase 3: integrate every row of every cell into K[(row * NQ + l) * CP + cell];
  // contributions of cells outside the mesh (partial tiles) are zero.  `stiff`
  // holds the nodal values the constant-coefficient gradient terms act on
  // (component 0 = c for the mu row, component 2 + i = eta_i for the eta rows).
  // With the grain cut-off (CUT) the row of a grain absent on the cell is zero
  // (do_vmult_range_no_template / do_evaluate_nonlinear_residual_nt,
  // operator_sintering_generic.h:456-537, :1008-1081, assemble the relevant
  // grains' rows only).  ADV: the eta_i row of a grain with a velocity on the
  // cell gains the flux -v_i eta_i (operator_sintering_generic.h:1015-1036,
  // :167-177), eta_i interpolated from the same nodal values `stiff` holds;
  // warps in which no cell of the row moves keep the value-only integration.
  // tc_b (packed pairs only): the tile of lane y, whose cells outside the
  // mesh are zeroed lane by lane.
  template <int DIM, int G, typename R, bool CUT = false, bool ADV = false>
  __device__ __forceinline__ void phase_integrate(const PhysR<R> &p, const Grid &g, const CellConsts<DIM, R> &k,
                                                  const TileCoord &tc, const R *P, const R *stiff, R *K,
                                                  unsigned m = ~0u, const R *vel = nullptr,
                                                  const unsigned char *has = nullptr,
                                                  const TileCoord *tc_b = nullptr)
  {
    using T            = Tile<DIM>;
    constexpr int NQ   = 1 << DIM;
    constexpr int C    = G + 2;
    constexpr int NGRP = T::THREADS / T::CELLS;
    // In 3D with fewer rows than thread groups, the c row (the only one with
    // a point-dependent flux, the longest) is shared by two groups, one per
    // layer of local nodes (z bit 0 / 1): C + 1 tasks instead of C rows.
    constexpr bool SPLIT0 = DIM == 3 && C + 1 <= NGRP;
    constexpr int  NTASK  = C + (SPLIT0 ? 1 : 0);
    const int     cell = threadIdx.x % T::CELLS;
    const int     b0   = cell_box_base<DIM>(cell);
    const bool    in   = cell_in_mesh<DIM>(cell, tc, g);
    const bool    in_b = tc_b ? cell_in_mesh<DIM>(cell, *tc_b, g) : in;
    for (int task = threadIdx.x / T::CELLS; task < NTASK; task += NGRP)
      {
        const int row = SPLIT0 ? (task < 2 ? 0 : task - 1) : task;
        if constexpr (SPLIT0)
          if (task < 2)
            {
              if (task == 0)
                integrate_c_row_half<0>(P, k, cell, in, in_b, K);
              else
                integrate_c_row_half<1>(P, k, cell, in, in_b, K);
              continue;
            }
        bool keep = in;
        if constexpr (CUT)
          if (row >= 2)
            {
              keep = keep && ((m >> (row - 2)) & 1u) != 0u;
              if (!__any_sync(0xffffffffu, keep))
                {
#pragma unroll
                  for (int l = 0; l < NQ; ++l)
                    K[(row * NQ + l) * T::CP + cell] = R(0);
                  continue;
                }
            }
        R r[NQ];
        if (row == 0)
          {
            R v[NQ], gg[DIM][NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q)
              {
                v[q] = P[(0 * NQ + q) * T::CELLS + cell];
#pragma unroll
                for (int d = 0; d < DIM; ++d)
                  gg[d][q] = P[((1 + d) * NQ + q) * T::CELLS + cell];
              }
            cell_integrate_vg<DIM>(v, gg, k, r);
          }
        else if (ADV && row >= 2 && __any_sync(0xffffffffu, has[(row - 2) * T::CELLS + cell] != 0))
          {
            R v[NQ], u[NQ], gg[DIM][NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q)
              {
                v[q] = P[((DIM + row) * NQ + q) * T::CELLS + cell];
#pragma unroll
                for (int d = 0; d < DIM; ++d)
                  gg[d][q] = R(0);
              }
            cell_nodes<DIM>(stiff + row * T::BOXS, b0, u);
            const int it = (row - 2) * T::CELLS + cell;
            if (has[it])
              {
                R e[NQ];
                cell_values<DIM>(u, k, e);
#pragma unroll
                for (int q = 0; q < NQ; ++q)
                  {
                    R dq[3], vq[DIM];
                    adv_offset<DIM>(k, g, q, dq);
                    adv_velocity<DIM>(vel, it, dq, vq);
#pragma unroll
                    for (int d = 0; d < DIM; ++d)
                      gg[d][q] = -(vq[d] * e[q]);
                  }
              }
            cell_integrate_vg<DIM>(v, gg, k, r);
            cell_stiffness_add<DIM, 1>(u, g, r);
          }
        else
          {
            const int res = DIM + row; // mu row: DIM + 1, eta_i row (row = 2 + i): DIM + 2 + i
            R         v[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q)
              v[q] = P[(res * NQ + q) * T::CELLS + cell];
            cell_integrate_v<DIM>(v, k, r);
            R u[NQ];
            cell_nodes<DIM>(stiff + (row == 1 ? 0 : row) * T::BOXS, b0, u);
            if (row == 1)
              cell_stiffness_add<DIM, 0>(u, g, r);
            else
              cell_stiffness_add<DIM, 1>(u, g, r);
          }
        // a branch, not a select per value: in tiles inside the mesh every
        // cell keeps its row
        if (keep && in_b)
          {
#pragma unroll
            for (int l = 0; l < NQ; ++l)
              K[(row * NQ + l) * T::CP + cell] = r[l];
          }
        else
          {
#pragma unroll
            for (int l = 0; l < NQ; ++l)
              K[(row * NQ + l) * T::CP + cell] = lane_keep(r[l], keep, in_b);
          }
      }
  }

  // Grain-cut-off mask of local cell `cell` of tile tc (one bit per grain,
  // n[0] x n[1] x n[2] cells in lexicographic order); cells outside the mesh
  // have no relevant grain.
  template <int DIM>
  __device__ __forceinline__ unsigned cell_mask(const uint16_t *__restrict__ mask, const Grid &g,
                                                const TileCoord &tc, int cell)
  {
    using T      = Tile<DIM>;
    const int cx = cell % T::TX, cy = (cell / T::TX) % T::TY, cz = cell / (T::TX * T::TY);
    const int i = tc.o[0] + cx, j = tc.o[1] + cy, k = DIM == 3 ? tc.o[2] + cz : 0;
    if (i >= g.n[0] || j >= g.n[1] || (DIM == 3 && k >= g.n[2]))
      return 0u;
    return mask[i + (long long)g.n[0] * (j + (long long)g.n[1] * k)];
  }

  // Cell mask m (bits = grains of the full operator) in the numbering of a
  // tile's compacted grain list gl: bit k set when grain gl[k] is relevant.
  template <int G>
  __device__ __forceinline__ unsigned local_mask(unsigned m, unsigned long long gl)
  {
    unsigned r = 0;
#pragma unroll
    for (int kk = 0; kk < G; ++kk)
      r |= ((m >> unsigned((gl >> (4 * kk)) & 15ull)) & 1u) << kk;
    return r;
  }

  template <int DIM, int G, bool TENS, bool JVP, bool HIST, bool ADV = false>
  struct ThreePhaseSmem
  {
    using T                     = Tile<DIM>;
    using FM                    = FieldMap<DIM, G, TENS, JVP, HIST>;
    static constexpr int C      = G + 2;
    static constexpr int NQ     = 1 << DIM;
    static constexpr int BOXES  = 2 * C * T::BOXS;                 // both inputs of one tile
    static constexpr int F_SIZE = FM::NSLOT * T::CELLS;            // point fields (K aliases it)
    static constexpr int P_SIZE = (DIM + 2 + G) * NQ * T::CELLS;   // point results
    static constexpr int K_SIZE = C * NQ * T::CP;
    static_assert(K_SIZE <= F_SIZE, "node contributions must fit in the point-field buffer");
    // staged advection coefficients (adv_stage): 6 values and one flag byte
    // per (grain, cell); the flags are counted in 4-byte elements
    static constexpr int ADV_VEL = ADV ? 6 * G * T::CELLS : 0;
    static constexpr int ADV_HAS = ADV ? (G * T::CELLS + 3) / 4 : 0;
    // elements: the JVP double-buffers its boxes, the residual does not
    static constexpr int TOTAL = (JVP ? 2 : 1) * BOXES + F_SIZE + P_SIZE + ADV_VEL + ADV_HAS;
  };

  // -------------------------------------------------------------------------
  // Jacobian-vector product: dst = J(lin) src.
  // SinteringOperatorGenericQuad::operator() (operator_sintering_generic.h:101-190)
  // inside do_vmult_range (:539-577), with the linearisation point evaluated
  // from the nodal state instead of a quadrature-point cache.  Persistent and
  // software pipelined: block b handles tiles b, b + grid, ...; the node boxes
  // of the next tile are copied (cp.async) into the second half of a double
  // buffer while the current tile is computed.
  // Two resident blocks per SM (<= 128 registers) unless the 3D FP64 grain
  // state of large G would spill (one block, up to 255 registers); the light
  // 2D FP32 product runs three (<= 85 registers), and the grain cut-off's
  // G = 0 class (c and mu only) four (<= 64 registers).
  template <int DIM, int G, typename R>
  constexpr int jvp_blocks_per_sm()
  {
    return G == 0 ? 4 : (DIM == 3 && sizeof(R) == 8 && G > 5) ? 1 : (DIM == 2 && sizeof(R) == 4) ? 3 : 2;
  }
  template <int DIM, int G>
  constexpr int residual_blocks_per_sm()
  {
    return G == 0 ? 4 : (DIM == 3 && G > 5) ? 1 : 2;
  }

  // CUT: grain cut-off.  The kernel instantiated for G grains runs over the
  // tiles of class G, ct.tiles[ct.range[G] .. ct.range[G + 1]), on their
  // compacted components (c, mu and the tile's G grains); a cell lacking one
  // of the tile's grains treats it as absent.  The tile ids, grain lists and
  // masks of the next tile are read one tile ahead, so their latency hides
  // behind the current tile.
  // ADV: with the advection terms of the grains' rigid-body velocities.
  template <int DIM, int G, bool TENS, typename R, bool CUT, bool ADV = false>
  __global__ void __launch_bounds__(Tile<DIM>::THREADS, jvp_blocks_per_sm<DIM, G, R>())
    jvp_kernel(const Grid g, const Phys ph, const R *__restrict__ lin, const R *__restrict__ src,
               R *__restrict__ dst, R *__restrict__ partial, const CutTiles ct, const AdvData adv)
  {
    using T  = Tile<DIM>;
    using SM = ThreePhaseSmem<DIM, G, TENS, true, false, ADV>;
    constexpr int C = G + 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *s_buf = reinterpret_cast<R *>(smem_raw); // 2 x BOXES
    R *F     = s_buf + 2 * SM::BOXES;
    R *P     = F + SM::F_SIZE;
    R *K     = F; // aliases the point fields, dead after phase 2
    R *A_vel = P + SM::P_SIZE;
    unsigned char *A_has = reinterpret_cast<unsigned char *>(A_vel + SM::ADV_VEL);

    const PhysR<R>           p(ph);
    const CellConsts<DIM, R> k(g);
    const NodePlan<DIM>      np(g);
    const int                cell = threadIdx.x % T::CELLS;
    const long long          i0   = CUT ? (long long)ct.range[G] : 0;
    const long long          i1   = CUT ? (long long)ct.range[G + 1] : g.n_tiles;
    long long                idx  = i0 + blockIdx.x;
    // node boxes of both inputs of tile tcx into buffer bb
    auto prefetch = [&](R *bb, const TileCoord &tcx, unsigned long long glx) {
      if (tile_interior<DIM>(g, tcx))
        {
          const long long n0 = tile_node0(g, tcx);
          load_box_async_interior<DIM>(bb, lin, C, g, np, n0, glx, CUT);
          load_box_async_interior<DIM>(bb + C * T::BOXS, src, C, g, np, n0, glx, CUT);
        }
      else
        {
          const BoxNode<DIM> bn(g, tcx);
          load_box_async<DIM>(bb, lin, C, g, bn, glx, CUT);
          load_box_async<DIM>(bb + C * T::BOXS, src, C, g, bn, glx, CUT);
        }
    };
    // current and next tile: id, grain list, union mask, this thread's cell mask
    long long          tile = 0, t_next = 0;
    unsigned long long gl = 0, gl_next = 0;
    unsigned           tm = 0, tm_next = 0, m_glob = ~0u, m_glob_next = ~0u;
    if constexpr (CUT)
      {
        if (idx < i1)
          {
            tile = ct.tiles[idx];
            gl   = ct.tile_grains[idx];
            tm   = ct.tile_mask[idx];
          }
        if (idx + gridDim.x < i1)
          {
            t_next  = ct.tiles[idx + gridDim.x];
            gl_next = ct.tile_grains[idx + gridDim.x];
            tm_next = ct.tile_mask[idx + gridDim.x];
          }
      }
    else
      tile = idx;
    if (idx < i1)
      {
        const TileCoord tc0 = tile_coord_of<DIM>(g, tile);
        prefetch(s_buf, tc0, gl);
        if constexpr (CUT)
          m_glob = cell_mask<DIM>(ct.cell_mask, g, tc0, cell);
      }
    cp_async_commit();
    for (int it = 0; idx < i1; ++it, idx += gridDim.x)
      {
        const long long nidx = idx + gridDim.x;
        R              *nb   = s_buf + ((it + 1) & 1) * SM::BOXES;
        long long       t_nn = 0; // the tile after next (CUT)
        unsigned long long gl_nn = 0;
        unsigned           tm_nn = 0;
        if (nidx < i1)
          {
            const long long next = CUT ? t_next : nidx;
            const TileCoord tcn  = tile_coord_of<DIM>(g, next);
            prefetch(nb, tcn, gl_next);
            if constexpr (CUT)
              {
                m_glob_next = cell_mask<DIM>(ct.cell_mask, g, tcn, cell);
                if (nidx + gridDim.x < i1)
                  {
                    t_nn  = ct.tiles[nidx + gridDim.x];
                    gl_nn = ct.tile_grains[nidx + gridDim.x];
                    tm_nn = ct.tile_mask[nidx + gridDim.x];
                  }
              }
          }
        cp_async_commit();
        cp_async_wait<1>(); // this tile's group has landed (only the prefetch may be pending)
        __syncthreads();
        const TileCoord tc = tile_coord_of<DIM>(g, tile);
        const R        *cb = s_buf + (it & 1) * SM::BOXES;
        const unsigned  m  = CUT ? local_mask<G>(m_glob, gl) : ~0u;
        if constexpr (ADV)
          adv_stage<DIM, G, R, CUT>(adv, g, tc, gl, A_vel, A_has);
        phase_evaluate<DIM, G, TENS, true, false, R, CUT>(cb, cb + C * T::BOXS, F, k, m);
        __syncthreads();
        jvp_point<DIM, G, TENS, R>(p, F, P, threadIdx.x / T::CELLS, cell, m);
        if constexpr (ADV)
          {
            using FM = FieldMap<DIM, G, TENS, true, false>;
            advect_c_point<DIM, G, R, CUT>(k, g, F, FM::base(FM::src_c), P, threadIdx.x / T::CELLS, cell, m, A_vel,
                                           A_has);
          }
        __syncthreads();
        phase_integrate<DIM, G, R, CUT, ADV>(p, g, k, tc, P, cb + C * T::BOXS, K, m, A_vel, A_has);
        __syncthreads();
        if (tile_interior<DIM>(g, tc))
          sum_and_store_interior<DIM>(K, C, g, tc.linear, np, tile_node0(g, tc), dst, partial, gl, CUT, ct.c_all, tm);
        else
          sum_and_store<DIM>(K, C, g, tc, BoxNode<DIM>(g, tc), dst, partial, gl, CUT, ct.c_all, tm);
        // No further barrier: the next tile's prefetch writes the other box
        // buffer, whose last readers (this tile's phases 1 and 3) passed the
        // barrier after phase 3, and K (aliasing F) is next written in phase
        // 1, after the barrier that follows the next cp.async wait.
        if constexpr (CUT)
          {
            tile    = t_next;
            gl      = gl_next;
            tm      = tm_next;
            m_glob  = m_glob_next;
            t_next  = t_nn;
            gl_next = gl_nn;
            tm_next = tm_nn;
          }
        else
          tile = nidx;
      }
    cp_async_wait<0>();
  }

  // -------------------------------------------------------------------------
  // FP32 Jacobian-vector product on tile pairs.  sm_100 executes FP32 add,
  // multiply and fused multiply-add on two values held in a 64-bit register
  // pair with one instruction (FADD2 / FMUL2 / FFMA2); the FP32 product is
  // bound by instruction issue, so the block computes tiles 2j and 2j + 1
  // together: every shared-memory value is a pair (lane x of tile 2j, lane y
  // of tile 2j + 1), phases 1-3 run once on F2 for both tiles, and the node
  // sums are stored per lane.  Each lane rounds exactly as the scalar FP32
  // arithmetic of the same expression does.  Full operator only (no grain
  // cut-off, no advection: those keep jvp_kernel); shared memory and
  // registers as the FP64 product.
  // CUT (G = 0 only): the grain cut-off's class of tiles without a relevant
  // grain, ct.tiles[ct.range[0] .. ct.range[1]), on c and mu; their owned
  // nodes get zero grain rows, as jvp_kernel's class-0 instance writes them.
  // Resident blocks per SM: as the FP64 product (pairs take the FP64 product's
  // registers), but three for the class without grains, whose pairs need
  // ~70 registers (four blocks would cap them at 64 and spill).
  template <int DIM, int G>
  constexpr int jvp_pair_blocks_per_sm()
  {
    return G == 0 ? 3 : jvp_blocks_per_sm<DIM, G, double>();
  }

  template <int DIM, int G, bool TENS, bool CUT = false>
  __global__ void __launch_bounds__(Tile<DIM>::THREADS, jvp_pair_blocks_per_sm<DIM, G>())
    jvp_pair_kernel(const Grid g, const Phys ph, const float *__restrict__ lin, const float *__restrict__ src,
                    float *__restrict__ dst, float *__restrict__ partial, const CutTiles ct)
  {
    static_assert(!CUT || G == 0, "the cut-off pair kernel serves the class without grains");
    using T  = Tile<DIM>;
    using SM = ThreePhaseSmem<DIM, G, TENS, true, false, false>;
    constexpr int C = G + 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    F2 *s_buf = reinterpret_cast<F2 *>(smem_raw); // 2 x BOXES pairs
    F2 *F     = s_buf + 2 * SM::BOXES;
    F2 *P     = F + SM::F_SIZE;
    F2 *K     = F; // aliases the point fields, dead after phase 2

    const PhysR<F2>           p(ph);
    const CellConsts<DIM, F2> k(g);
    const NodePlan<DIM>       np(g);
    const int                 cell   = threadIdx.x % T::CELLS;
    // the tiles served: all of them, or the class-0 list of the cut-off
    const long long           i0     = CUT ? (long long)ct.range[0] : 0;
    const long long           nt     = CUT ? (long long)ct.range[1] - i0 : g.n_tiles;
    const long long           npairs = (nt + 1) / 2;
    auto tile_id = [&](long long i) -> long long { return CUT ? (long long)ct.tiles[i0 + i] : i; };
    long long                 idx    = blockIdx.x;
    // node boxes of both inputs of the tiles of pair j into buffer bb (a
    // missing second tile leaves its lane stale: computed, never stored)
    auto prefetch = [&](F2 *bb, long long j) {
#pragma unroll
      for (int lane = 0; lane < 2; ++lane)
        {
          if (2 * j + lane >= nt)
            break;
          const long long tile = tile_id(2 * j + lane);
          const TileCoord tcx  = tile_coord_of<DIM>(g, tile);
          float          *fb  = reinterpret_cast<float *>(bb) + lane;
          if (tile_interior<DIM>(g, tcx))
            {
              const long long n0 = tile_node0(g, tcx);
              load_box_async_interior<DIM, float, 2>(fb, lin, C, g, np, n0);
              load_box_async_interior<DIM, float, 2>(fb + 2 * C * T::BOXS, src, C, g, np, n0);
            }
          else
            {
              const BoxNode<DIM> bn(g, tcx);
              load_box_async<DIM, float, 2>(fb, lin, C, g, bn);
              load_box_async<DIM, float, 2>(fb + 2 * C * T::BOXS, src, C, g, bn);
            }
        }
    };
    if (idx < npairs)
      prefetch(s_buf, idx);
    cp_async_commit();
    for (int it = 0; idx < npairs; ++it, idx += gridDim.x)
      {
        const long long nidx = idx + gridDim.x;
        if (nidx < npairs)
          prefetch(s_buf + ((it + 1) & 1) * SM::BOXES, nidx);
        cp_async_commit();
        cp_async_wait<1>(); // this pair's group has landed (only the prefetch may be pending)
        __syncthreads();
        const bool      has_b  = 2 * idx + 1 < nt;
        const long long tile_a = tile_id(2 * idx), tile_b = has_b ? tile_id(2 * idx + 1) : tile_a;
        const TileCoord tca    = tile_coord_of<DIM>(g, tile_a);
        const TileCoord tcb    = tile_coord_of<DIM>(g, tile_b);
        const F2       *cb     = s_buf + (it & 1) * SM::BOXES;
        phase_evaluate<DIM, G, TENS, true, false, F2, false>(cb, cb + C * T::BOXS, F, k);
        __syncthreads();
        jvp_point<DIM, G, TENS, F2>(p, F, P, threadIdx.x / T::CELLS, cell);
        __syncthreads();
        phase_integrate<DIM, G, F2, false, false>(p, g, k, tca, P, cb + C * T::BOXS, K, ~0u, nullptr, nullptr,
                                                  &tcb);
        __syncthreads();
#pragma unroll
        for (int lane = 0; lane < 2; ++lane)
          {
            if (lane == 1 && !has_b)
              break;
            const TileCoord &tc = lane ? tcb : tca;
            const float     *kf = reinterpret_cast<const float *>(K) + lane;
            // CUT: c and mu are components 0 and 1 of the c_all-component
            // layout; no grain is relevant on the tile (union mask 0)
            if (tile_interior<DIM>(g, tc))
              sum_and_store_interior<DIM, float, 2>(kf, C, g, tc.linear, np, tile_node0(g, tc), dst, partial, 0, CUT,
                                                    ct.c_all, 0u);
            else
              sum_and_store<DIM, float, 2>(kf, C, g, tc, BoxNode<DIM>(g, tc), dst, partial, 0, CUT, ct.c_all, 0u);
          }
      }
    cp_async_wait<0>();
  }

  // -------------------------------------------------------------------------
  // Nonlinear residual: dst = R(src), SinteringOperatorGenericResidualQuad
  // (operator_sintering_generic.h:254-308) with the history of
  // do_evalute_history (:927-975) for WTD == 2: the weighted sum of the old
  // solutions is formed at the nodes while staging and evaluated at the points.
  // CUT: the kernel for G grains runs over the tiles of class G on their
  // compacted components, as the Jacobian product does.
  // ADV: with the advection terms of the grains' rigid-body velocities.
  template <int DIM, int G, bool TENS, int WTD, bool CUT, bool ADV = false>
  __global__ void __launch_bounds__(Tile<DIM>::THREADS, residual_blocks_per_sm<DIM, G>())
    residual_kernel(const Grid g, const Phys ph, const double *__restrict__ src, const double *__restrict__ h0,
                    const double *__restrict__ h1, const double *__restrict__ h2, double *__restrict__ dst,
                    double *__restrict__ partial, const CutTiles ct, const AdvData adv)
  {
    using R  = double;
    using T  = Tile<DIM>;
    using SM = ThreePhaseSmem<DIM, G, TENS, false, WTD == 2, ADV>;
    constexpr int C = G + 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *s_u = reinterpret_cast<R *>(smem_raw);
    R *s_h = s_u + C * T::BOXS;
    R *F   = s_u + SM::BOXES;
    R *P   = F + SM::F_SIZE;
    R *K   = F;
    R *A_vel = P + SM::P_SIZE;
    unsigned char *A_has = reinterpret_cast<unsigned char *>(A_vel + SM::ADV_VEL);

    const PhysR<R>           p(ph);
    const CellConsts<DIM, R> k(g);
    const NodePlan<DIM>      np(g);
    const long long          i0 = CUT ? (long long)ct.range[G] : 0;
    const long long          i1 = CUT ? (long long)ct.range[G + 1] : g.n_tiles;
    for (long long idx = i0 + blockIdx.x; idx < i1; idx += gridDim.x)
      {
        const long long          tile = CUT ? (long long)ct.tiles[idx] : idx;
        const unsigned long long gl   = CUT ? ct.tile_grains[idx] : 0ull;
        const unsigned           tm   = CUT ? ct.tile_mask[idx] : 0u;
        const TileCoord          tc   = tile_coord_of<DIM>(g, tile);
        const bool               interior = tile_interior<DIM>(g, tc);
        const long long          node0    = tile_node0(g, tc);
        const unsigned m = CUT ? local_mask<G>(cell_mask<DIM>(ct.cell_mask, g, tc, threadIdx.x % T::CELLS), gl) : ~0u;
        // this thread's box node: in an interior tile it exists and reads itself
        bool      inside = true;
        long long lidx   = node0 + np.off;
        if (!interior)
          {
            const BoxNode<DIM> bn(g, tc);
            inside = bn.inside;
            lidx   = bn.lidx;
          }
        if (np.active)
          for (int comp = np.grp; comp < C; comp += T::NG)
            {
              R v = R(0), hv = R(0);
              if (inside)
                {
                  const long long off = (CUT ? comp_of(comp, gl) : comp) * g.ld + lidx;
                  v                   = src[off];
                  if (ph.hooks.perturb) // the residual's perturbation hook: src + a x
                    v = src[off] + ph.hooks.perturb_scale * ph.hooks.perturb[off];
                  // sum_i w_{i+1} u_old_i at the nodes (generic.h:947-966); mu has no history
                  if (WTD == 2 && comp != 1)
                    {
                      hv = h0[off] * ph.w_hist[0];
                      if (ph.order > 1)
                        hv += h1[off] * ph.w_hist[1];
                      if (ph.order > 2)
                        hv += h2[off] * ph.w_hist[2];
                    }
                }
              s_u[comp * T::BOXS + np.sb] = v;
              if constexpr (WTD == 2)
                s_h[comp * T::BOXS + np.sb] = hv;
            }
        if constexpr (ADV)
          adv_stage<DIM, G, R, CUT>(adv, g, tc, gl, A_vel, A_has);
        __syncthreads();
        phase_evaluate<DIM, G, TENS, false, WTD == 2, R, CUT>(s_u, s_h, F, k, m);
        __syncthreads();
        residual_point<DIM, G, TENS, WTD, R>(p, F, P, threadIdx.x / T::CELLS, threadIdx.x % T::CELLS, m);
        if constexpr (ADV)
          {
            using FM = FieldMap<DIM, G, TENS, false, WTD == 2>;
            advect_c_point<DIM, G, R, CUT>(k, g, F, FM::base(FM::lin_c), P, threadIdx.x / T::CELLS,
                                           threadIdx.x % T::CELLS, m, A_vel, A_has);
          }
        __syncthreads();
        phase_integrate<DIM, G, R, CUT, ADV>(p, g, k, tc, P, s_u, K, m, A_vel, A_has);
        __syncthreads();
        if (interior)
          sum_and_store_interior<DIM>(K, C, g, tc.linear, np, node0, dst, partial, gl, CUT, ct.c_all, tm, &ph.hooks);
        else
          sum_and_store<DIM>(K, C, g, tc, BoxNode<DIM>(g, tc), dst, partial, gl, CUT, ct.c_all, tm, &ph.hooks);
        // no barrier: the next tile's staging writes the boxes, read last in
        // phase 3 before the barrier above; K (aliasing F) is next written in
        // phase 1, after the barrier that follows the staging
      }
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
  template <int DIM, int G, bool TENS, bool ADV = false>
  struct DiagLayout
  {
    static constexpr int NOUT  = G + 4;
    static constexpr int NADV  = ADV ? G * DIM : 0; // the grains' velocities at the point
    static constexpr int NCOEF = DIM * DIM + DIM + DIM * DIM + 1 + G + NADV;
  };

  // CUT: the grains absent on a cell (mask bit clear) have zero values there
  // and no Allen-Cahn diagonal contribution from it (preconditioners.h:787-817).
  // ADV: the advection terms of the preconditioner's operators
  // (precondition_advection_ch / _ac, operator_sintering_generic.h:800-850):
  // J_cc gains -(phi_l sum_i v_i, grad phi_l) and grain i's diagonal
  // -(phi_l v_i, grad phi_l), with the velocities of the current table.
  template <int DIM, int G, bool TENS, bool CUT, bool ADV = false>
  __global__ void __launch_bounds__(Tile<DIM>::THREADS)
    diag_kernel(const Grid g, const Phys ph, const double *__restrict__ lin, double *__restrict__ dst,
                double *__restrict__ partial, const uint16_t *__restrict__ mask, const AdvData adv)
  {
    using R          = double;
    using T          = Tile<DIM>;
    using LY         = DiagLayout<DIM, G, TENS, ADV>;
    constexpr int C  = G + 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *s_lin  = reinterpret_cast<R *>(smem_raw);
    R *s_coef = s_lin + C * T::BOXS;
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
    const unsigned   gmask = CUT ? cell_mask<DIM>(mask, g, tc, cell) : ~0u;

    {
      R c, gc[DIM], mu_unused, gmu[DIM];
      eval_vg<DIM>(s_lin, b0, w, c, gc);
      eval_vg<DIM>(s_lin + T::BOXS, b0, w, mu_unused, gmu);
      R eta[G];
      R geta[G][DIM];
#pragma unroll
      for (int i = 0; i < G; ++i)
        {
          eval_vg<DIM>(s_lin + (2 + i) * T::BOXS, b0, w, eta[i], geta[i]);
          if (CUT && ((gmask >> i) & 1u) == 0u)
            {
              eta[i] = R(0);
#pragma unroll
              for (int d = 0; d < DIM; ++d)
                geta[i][d] = R(0);
            }
        }
      R *cf = s_coef + threadIdx.x * LY::NCOEF;
      // mobility matrix (M grad mu = apply_M(grad mu)) in one pass over the
      // grain pairs; absent grains (CUT) enter with zero values
      {
        R Mm[DIM][DIM];
        mobility_matrix<DIM, G, TENS>(p, c, eta, gc, geta, Mm);
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int b = 0; b < DIM; ++b)
            cf[a * DIM + b] = Mm[a][b];
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
      if constexpr (ADV)
        {
          // velocity of every grain at this thread's point (zero without a segment)
          R        *vc = cf + 2 * DIM * DIM + DIM + 1 + G;
          int       cc[3];
          const int q  = threadIdx.x & (T::NQ - 1);
          const bool in = cell_global<DIM>(cell, tc, g, cc);
          const long long n_cells = (long long)g.n[0] * g.n[1] * g.n[2];
          const long long lin_cell = cc[0] + (long long)g.n[0] * (cc[1] + (long long)g.n[1] * cc[2]);
          const double gp0 = 0.5 - 0.5 / sqrt(3.0), gp1 = 0.5 + 0.5 / sqrt(3.0);
#pragma unroll 1
          for (int i = 0; i < G; ++i)
            {
              int s = -1;
              if (in && (!CUT || ((gmask >> i) & 1u)))
                {
                  s = adv.cell_segments[i * n_cells + lin_cell];
                  if (s >= adv.n_segments)
                    s = -1;
                }
              R v[3] = {R(0), R(0), R(0)};
              if (s >= 0)
                {
                  const double *d    = adv.segments + 9 * (long long)s;
                  double        r[3] = {0.0, 0.0, 0.0};
#pragma unroll
                  for (int e = 0; e < DIM; ++e)
                    r[e] = adv.origin[e] + (cc[e] + (((q >> e) & 1) ? gp1 : gp0)) * g.h[e] - d[6 + e];
                  v[0] = d[0] + d[4] * r[2] - d[5] * r[1];
                  v[1] = d[1] + d[5] * r[0] - d[3] * r[2];
                  v[2] = d[2] + d[3] * r[1] - d[4] * r[0];
                }
#pragma unroll
              for (int e = 0; e < DIM; ++e)
                vc[i * DIM + e] = v[e];
            }
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
          if constexpr (ADV)
            {
              const R *vc = cf + 2 * DIM * DIM + DIM + 1 + G;
#pragma unroll
              for (int i = 0; i < G; ++i)
                {
                  R vd = R(0);
#pragma unroll
                  for (int e = 0; e < DIM; ++e)
                    vd += vc[i * DIM + e] * dphi[e];
                  acc[0] -= w.JxW * phi * vd;
                  acc[4 + i] -= w.JxW * phi * vd;
                }
            }
        }
#pragma unroll
      for (int i = 0; i < G; ++i)
        if (CUT && ((gmask >> i) & 1u) == 0u)
          acc[4 + i] = R(0);
#pragma unroll
      for (int k = 0; k < LY::NOUT; ++k)
        store_contrib<DIM>(s_con, k, acc[k], valid);
    }
    __syncthreads();
    sum_and_store<DIM>(s_con, LY::NOUT, g, tc, bn, dst, partial);
  }
} // namespace sint
