// Per-cell sum factorisation for the three-phase cell kernels.
//
// Phase 1 (evaluation): one thread per (cell, component) interpolates the
// cell's 2^dim nodal values to all 2^dim Gauss points and, for components
// whose gradient is needed, the gradient.  A Q1 gradient component d depends
// only on the point coordinates in the other directions, so it has 2^(dim-1)
// distinct values per cell; only those are stored ("gradient slots").
// Phase 3 (integration): one thread per (cell, residual row) contracts the
// row's point values (and, for the c row, point fluxes) with the test
// functions by the transposed sum factorisation and adds the exact element
// stiffness term for rows whose gradient flux has a constant coefficient.
//
// Point index q = qx + 2 qy (+ 4 qz); 1D Gauss point coordinates on [0, 1]:
// x_0 = 1/2 - 1/(2 sqrt 3), x_1 = 1/2 + 1/(2 sqrt 3); 1D shape functions
// phi_0(x) = 1 - x, phi_1(x) = x, so phi_l(x_q) = (l == q) ? x_1 : x_0.
#pragma once

#include "sint_common.cuh"

namespace sint
{
  template <int DIM, typename R>
  struct CellConsts
  {
    R x0, x1;   // Gauss point coordinates
    R nx1;      // -x1
    R ih[DIM];  // 1 / h
    R dih[DIM]; // (+1) / h: derivative of phi_1 (phi_0 has the negative)
    R JxW;

    __device__ __forceinline__ explicit CellConsts(const Grid &g)
    {
      const double s3 = 0.5 / 1.7320508075688772935274463415058723669428;
      x0              = R(0.5 - s3);
      x1              = R(0.5 + s3);
      nx1             = R(-(0.5 + s3));
      double jxw      = 1.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        {
          ih[d]  = R(1.0 / g.h[d]);
          dih[d] = ih[d];
          jxw *= 0.5 * g.h[d];
        }
      JxW = R(jxw);
    }
  };

  // number of stored slots of one evaluated component
  template <int DIM>
  struct Slots
  {
    static constexpr int NQ  = 1 << DIM;
    static constexpr int NG1 = NQ / 2;          // distinct values of one gradient component
    static constexpr int V   = NQ;              // value only
    static constexpr int VG  = NQ + DIM * NG1; // value + gradient
  };

  // gradient slot of point q for direction d
  template <int DIM>
  __device__ __forceinline__ int grad_slot(int d, int q)
  {
    if constexpr (DIM == 3)
      return d == 0 ? (q >> 1) : (d == 1 ? ((q & 1) | ((q >> 1) & 2)) : (q & 3));
    else
      return d == 0 ? (q >> 1) : (q & 1);
  }

  // the cell's nodal values of one component from the staged box
  template <int DIM, typename R>
  __device__ __forceinline__ void cell_nodes(const R *s, int b0, R (&u)[1 << DIM])
  {
    using T = Tile<DIM>;
#pragma unroll
    for (int l = 0; l < (1 << DIM); ++l)
      u[l] = s[b0 + (l & 1) + T::SY * ((l >> 1) & 1) + (DIM == 3 ? T::SZ * ((l >> 2) & 1) : 0)];
  }

  // Phase 1, value + gradient: writes F[(base + slot) * CELLS + cell] for the
  // NQ values followed by DIM blocks of NG1 gradient slots.
  template <int DIM, typename R>
  __device__ __forceinline__ void cell_eval_vg(const R (&u)[1 << DIM], const CellConsts<DIM, R> &k, R *F, int base,
                                               int cell)
  {
    constexpr int CELLS = Tile<DIM>::CELLS;
    const R       xq[2] = {k.x0, k.x1};
    if constexpr (DIM == 3)
      {
        R vx[2][2][2], dxl[2][2];
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
#pragma unroll
          for (int ly = 0; ly < 2; ++ly)
            {
              const R u0 = u[2 * ly + 4 * lz], d = u[1 + 2 * ly + 4 * lz] - u0;
              dxl[lz][ly] = d;
#pragma unroll
              for (int qx = 0; qx < 2; ++qx)
                vx[lz][ly][qx] = u0 + xq[qx] * d;
            }
        R vxy[2][2][2], dyl[2][2], dxy[2][2];
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
          {
#pragma unroll
            for (int qx = 0; qx < 2; ++qx)
              {
                const R d = vx[lz][1][qx] - vx[lz][0][qx];
                dyl[lz][qx] = d;
#pragma unroll
                for (int qy = 0; qy < 2; ++qy)
                  vxy[lz][qy][qx] = vx[lz][0][qx] + xq[qy] * d;
              }
            const R dd = dxl[lz][1] - dxl[lz][0];
#pragma unroll
            for (int qy = 0; qy < 2; ++qy)
              dxy[lz][qy] = dxl[lz][0] + xq[qy] * dd;
          }
#pragma unroll
        for (int qy = 0; qy < 2; ++qy)
#pragma unroll
          for (int qx = 0; qx < 2; ++qx)
            {
              const R d = vxy[1][qy][qx] - vxy[0][qy][qx];
#pragma unroll
              for (int qz = 0; qz < 2; ++qz)
                F[(base + qx + 2 * qy + 4 * qz) * CELLS + cell] = vxy[0][qy][qx] + xq[qz] * d;
              F[(base + 8 + 8 + qx + 2 * qy) * CELLS + cell] = d * k.ih[2]; // d/dz at (qy, qx)
            }
#pragma unroll
        for (int qy = 0; qy < 2; ++qy)
          {
            const R dd = dxy[1][qy] - dxy[0][qy];
#pragma unroll
            for (int qz = 0; qz < 2; ++qz)
              F[(base + 8 + qy + 2 * qz) * CELLS + cell] = (dxy[0][qy] + xq[qz] * dd) * k.ih[0]; // d/dx at (qz, qy)
          }
#pragma unroll
        for (int qx = 0; qx < 2; ++qx)
          {
            const R dd = dyl[1][qx] - dyl[0][qx];
#pragma unroll
            for (int qz = 0; qz < 2; ++qz)
              F[(base + 8 + 4 + qx + 2 * qz) * CELLS + cell] = (dyl[0][qx] + xq[qz] * dd) * k.ih[1]; // d/dy at (qz, qx)
          }
      }
    else
      {
        R vx[2][2], dxl[2];
#pragma unroll
        for (int ly = 0; ly < 2; ++ly)
          {
            const R u0 = u[2 * ly], d = u[1 + 2 * ly] - u0;
            dxl[ly] = d;
#pragma unroll
            for (int qx = 0; qx < 2; ++qx)
              vx[ly][qx] = u0 + xq[qx] * d;
          }
#pragma unroll
        for (int qx = 0; qx < 2; ++qx)
          {
            const R d = vx[1][qx] - vx[0][qx];
#pragma unroll
            for (int qy = 0; qy < 2; ++qy)
              F[(base + qx + 2 * qy) * CELLS + cell] = vx[0][qx] + xq[qy] * d;
            F[(base + 4 + 2 + qx) * CELLS + cell] = d * k.ih[1]; // d/dy at qx
          }
        const R dd = dxl[1] - dxl[0];
#pragma unroll
        for (int qy = 0; qy < 2; ++qy)
          F[(base + 4 + qy) * CELLS + cell] = (dxl[0] + xq[qy] * dd) * k.ih[0]; // d/dx at qy
      }
  }

  // Phase 1, value only: F[(base + q) * CELLS + cell].
  template <int DIM, typename R>
  __device__ __forceinline__ void cell_eval_v(const R (&u)[1 << DIM], const CellConsts<DIM, R> &k, R *F, int base,
                                              int cell)
  {
    constexpr int CELLS = Tile<DIM>::CELLS;
    const R       xq[2] = {k.x0, k.x1};
    if constexpr (DIM == 3)
      {
        R vx[2][2][2];
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
#pragma unroll
          for (int ly = 0; ly < 2; ++ly)
            {
              const R u0 = u[2 * ly + 4 * lz], d = u[1 + 2 * ly + 4 * lz] - u0;
#pragma unroll
              for (int qx = 0; qx < 2; ++qx)
                vx[lz][ly][qx] = u0 + xq[qx] * d;
            }
        R vxy[2][2][2];
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
#pragma unroll
          for (int qx = 0; qx < 2; ++qx)
            {
              const R d = vx[lz][1][qx] - vx[lz][0][qx];
#pragma unroll
              for (int qy = 0; qy < 2; ++qy)
                vxy[lz][qy][qx] = vx[lz][0][qx] + xq[qy] * d;
            }
#pragma unroll
        for (int qy = 0; qy < 2; ++qy)
#pragma unroll
          for (int qx = 0; qx < 2; ++qx)
            {
              const R d = vxy[1][qy][qx] - vxy[0][qy][qx];
#pragma unroll
              for (int qz = 0; qz < 2; ++qz)
                F[(base + qx + 2 * qy + 4 * qz) * CELLS + cell] = vxy[0][qy][qx] + xq[qz] * d;
            }
      }
    else
      {
        R vx[2][2];
#pragma unroll
        for (int ly = 0; ly < 2; ++ly)
          {
            const R u0 = u[2 * ly], d = u[1 + 2 * ly] - u0;
#pragma unroll
            for (int qx = 0; qx < 2; ++qx)
              vx[ly][qx] = u0 + xq[qx] * d;
          }
#pragma unroll
        for (int qx = 0; qx < 2; ++qx)
          {
            const R d = vx[1][qx] - vx[0][qx];
#pragma unroll
            for (int qy = 0; qy < 2; ++qy)
              F[(base + qx + 2 * qy) * CELLS + cell] = vx[0][qx] + xq[qy] * d;
          }
      }
  }

  // Values at the NQ points in registers: vq[q] = sum_l phi_l(x_q) u_l, one
  // direction at a time.
  template <int DIM, typename R>
  __device__ __forceinline__ void cell_values(const R (&u)[1 << DIM], const CellConsts<DIM, R> &k,
                                              R (&vq)[1 << DIM])
  {
    constexpr int NQ = 1 << DIM;
    const R       xq[2] = {k.x0, k.x1};
    R             a[NQ];
#pragma unroll
    for (int l = 0; l < NQ; ++l)
      a[l] = u[l];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      {
        // a is indexed by point bits below d and node bits from d on
        R b[NQ];
#pragma unroll
        for (int i = 0; i < NQ; ++i)
          {
            const int lo = i & ~(1 << d), hi = i | (1 << d);
            b[i]         = a[lo] + xq[(i >> d) & 1] * (a[hi] - a[lo]);
          }
#pragma unroll
        for (int i = 0; i < NQ; ++i)
          a[i] = b[i];
      }
#pragma unroll
    for (int q = 0; q < NQ; ++q)
      vq[q] = a[q];
  }

  // 1D contraction of a point pair (a at x_0, b at x_1) with phi_l:
  // l = 0 -> x_1 a + x_0 b, l = 1 -> x_0 a + x_1 b.  With x_0 + x_1 = 1 both
  // share the difference: r_0 = b + x_1 (a - b), r_1 = a - x_1 (a - b) (three
  // operations instead of four).
  template <typename R>
  __device__ __forceinline__ void contract(const R a, const R b, const R x1, const R nx1, R &r0, R &r1)
  {
    const R d = a - b;
    r0        = b + x1 * d;
    r1        = a + nx1 * d;
  }
  // one output of the contraction: l = HZ
  template <int HZ, typename R>
  __device__ __forceinline__ R contract1(const R a, const R b, const R x1, const R nx1)
  {
    const R d = a - b;
    if constexpr (HZ == 0)
      return b + x1 * d;
    else
      return a + nx1 * d;
  }

  // Phase 3, full row: r_l = JxW sum_q (v_q phi_l(x_q) + g_q . grad phi_l(x_q)).
  template <int DIM, typename R>
  __device__ __forceinline__ void cell_integrate_vg(const R (&v)[1 << DIM], const R (&g)[DIM][1 << DIM],
                                                    const CellConsts<DIM, R> &k, R (&r)[1 << DIM])
  {
    if constexpr (DIM == 3)
      {
        // contract z: A (value-like incl. the z flux), BX, BY
        R A[2][2][2], BX[2][2][2], BY[2][2][2];
#pragma unroll
        for (int qy = 0; qy < 2; ++qy)
#pragma unroll
          for (int qx = 0; qx < 2; ++qx)
            {
              const int q0 = qx + 2 * qy, q1 = q0 + 4;
              const R   sz = (g[2][q0] + g[2][q1]) * k.dih[2];
              R         a0, a1;
              contract(v[q0], v[q1], k.x1, k.nx1, a0, a1);
              A[0][qy][qx] = a0 - sz;
              A[1][qy][qx] = a1 + sz;
              contract(g[0][q0], g[0][q1], k.x1, k.nx1, BX[0][qy][qx], BX[1][qy][qx]);
              contract(g[1][q0], g[1][q1], k.x1, k.nx1, BY[0][qy][qx], BY[1][qy][qx]);
            }
        // contract y
        R A2[2][2][2], BX2[2][2][2];
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
#pragma unroll
          for (int qx = 0; qx < 2; ++qx)
            {
              const R sy = (BY[lz][0][qx] + BY[lz][1][qx]) * k.dih[1];
              R       a0, a1;
              contract(A[lz][0][qx], A[lz][1][qx], k.x1, k.nx1, a0, a1);
              A2[lz][0][qx] = a0 - sy;
              A2[lz][1][qx] = a1 + sy;
              contract(BX[lz][0][qx], BX[lz][1][qx], k.x1, k.nx1, BX2[lz][0][qx], BX2[lz][1][qx]);
            }
        // contract x
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
#pragma unroll
          for (int ly = 0; ly < 2; ++ly)
            {
              const R sx = (BX2[lz][ly][0] + BX2[lz][ly][1]) * k.dih[0];
              R       a0, a1;
              contract(A2[lz][ly][0], A2[lz][ly][1], k.x1, k.nx1, a0, a1);
              r[2 * ly + 4 * lz]     = (a0 - sx) * k.JxW;
              r[1 + 2 * ly + 4 * lz] = (a1 + sx) * k.JxW;
            }
      }
    else
      {
        R A[2][2], BX[2][2];
#pragma unroll
        for (int qx = 0; qx < 2; ++qx)
          {
            const int q0 = qx, q1 = qx + 2;
            const R   sy = (g[1][q0] + g[1][q1]) * k.dih[1];
            R         a0, a1;
            contract(v[q0], v[q1], k.x1, k.nx1, a0, a1);
            A[0][qx] = a0 - sy;
            A[1][qx] = a1 + sy;
            contract(g[0][q0], g[0][q1], k.x1, k.nx1, BX[0][qx], BX[1][qx]);
          }
#pragma unroll
        for (int ly = 0; ly < 2; ++ly)
          {
            const R sx = (BX[ly][0] + BX[ly][1]) * k.dih[0];
            R       a0, a1;
            contract(A[ly][0], A[ly][1], k.x1, k.nx1, a0, a1);
            r[2 * ly]     = (a0 - sx) * k.JxW;
            r[1 + 2 * ly] = (a1 + sx) * k.JxW;
          }
      }
  }

  // Phase 3, full row in 3D, the half of the local nodes with z bit HZ: writes
  // r[l] for l = lx + 2 ly + 4 HZ only.  Two threads of a cell share a row
  // this way, each contracting z to its own node layer first.
  template <int HZ, typename R>
  __device__ __forceinline__ void cell_integrate_vg_half(const R (&v)[8], const R (&g)[3][8],
                                                         const CellConsts<3, R> &k, R (&r)[8])
  {
    R A[2][2], BX[2][2], BY[2][2];
#pragma unroll
    for (int qy = 0; qy < 2; ++qy)
#pragma unroll
      for (int qx = 0; qx < 2; ++qx)
        {
          const int q0 = qx + 2 * qy, q1 = q0 + 4;
          const R   sz = (g[2][q0] + g[2][q1]) * k.dih[2];
          const R   a  = contract1<HZ>(v[q0], v[q1], k.x1, k.nx1);
          A[qy][qx]    = HZ ? a + sz : a - sz;
          BX[qy][qx]   = contract1<HZ>(g[0][q0], g[0][q1], k.x1, k.nx1);
          BY[qy][qx]   = contract1<HZ>(g[1][q0], g[1][q1], k.x1, k.nx1);
        }
    R A2[2][2], BX2[2][2];
#pragma unroll
    for (int qx = 0; qx < 2; ++qx)
      {
        const R sy = (BY[0][qx] + BY[1][qx]) * k.dih[1];
        R       a0, a1;
        contract(A[0][qx], A[1][qx], k.x1, k.nx1, a0, a1);
        A2[0][qx] = a0 - sy;
        A2[1][qx] = a1 + sy;
        contract(BX[0][qx], BX[1][qx], k.x1, k.nx1, BX2[0][qx], BX2[1][qx]);
      }
#pragma unroll
    for (int ly = 0; ly < 2; ++ly)
      {
        const R sx = (BX2[ly][0] + BX2[ly][1]) * k.dih[0];
        R       a0, a1;
        contract(A2[ly][0], A2[ly][1], k.x1, k.nx1, a0, a1);
        r[2 * ly + 4 * HZ]     = (a0 - sx) * k.JxW;
        r[1 + 2 * ly + 4 * HZ] = (a1 + sx) * k.JxW;
      }
  }

  // Phase 3, value-only row: r_l = JxW sum_q v_q phi_l(x_q).
  template <int DIM, typename R>
  __device__ __forceinline__ void cell_integrate_v(const R (&v)[1 << DIM], const CellConsts<DIM, R> &k,
                                                   R (&r)[1 << DIM])
  {
    if constexpr (DIM == 3)
      {
        R A[2][2][2];
#pragma unroll
        for (int qy = 0; qy < 2; ++qy)
#pragma unroll
          for (int qx = 0; qx < 2; ++qx)
            contract(v[qx + 2 * qy], v[qx + 2 * qy + 4], k.x1, k.nx1, A[0][qy][qx], A[1][qy][qx]);
        R A2[2][2][2];
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
#pragma unroll
          for (int qx = 0; qx < 2; ++qx)
            contract(A[lz][0][qx], A[lz][1][qx], k.x1, k.nx1, A2[lz][0][qx], A2[lz][1][qx]);
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
#pragma unroll
          for (int ly = 0; ly < 2; ++ly)
            {
              R a0, a1;
              contract(A2[lz][ly][0], A2[lz][ly][1], k.x1, k.nx1, a0, a1);
              r[2 * ly + 4 * lz]     = a0 * k.JxW;
              r[1 + 2 * ly + 4 * lz] = a1 * k.JxW;
            }
      }
    else
      {
        R A[2][2];
#pragma unroll
        for (int qx = 0; qx < 2; ++qx)
          contract(v[qx], v[qx + 2], k.x1, k.nx1, A[0][qx], A[1][qx]);
#pragma unroll
        for (int ly = 0; ly < 2; ++ly)
          {
            R a0, a1;
            contract(A[ly][0], A[ly][1], k.x1, k.nx1, a0, a1);
            r[2 * ly]     = a0 * k.JxW;
            r[1 + 2 * ly] = a1 * k.JxW;
          }
      }
  }

  // r_l += coef (K u)_l with the exact element Laplacian K_lm = kx[l xor m],
  // coef kx taken from the grid's row coefficients (ROW 0: -kappa_c for the
  // mu row, 1: L kappa_p for the eta rows), so every term is one fused
  // multiply-add with a launch constant.
  template <int DIM, int ROW, typename R>
  __device__ __forceinline__ void cell_stiffness_add(const R (&u)[1 << DIM], const Grid &g, R (&r)[1 << DIM])
  {
#pragma unroll
    for (int l = 0; l < (1 << DIM); ++l)
      {
        R acc = r[l];
#pragma unroll
        for (int x = 0; x < (1 << DIM); ++x)
          acc += kst<R>(g, ROW, x) * u[l ^ x];
        r[l] = acc;
      }
  }
} // namespace sint
