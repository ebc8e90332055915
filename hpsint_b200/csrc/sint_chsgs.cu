// Matrix-based preconditioner of the Cahn-Hilliard block.
//
// hpsint's default BlockPreconditioner2 (sintering/preconditioners.h:1222-1283,
// block_0 = "ILU", preconditioner_parameters.h) assembles the Cahn-Hilliard
// block of the tangent (OperatorCahnHilliard::do_vmult_kernel,
// preconditioners.h:85-169, through MyMatrixFreeTools::compute_matrix,
// matrix_free/tools.h:29-175) and factorises it with ILU(0)
// (lac/preconditioners.h:607-1088); the grain block keeps the inverse
// diagonal.  On the GPU the triangular solves of a natural-order ILU are
// sequential, so this build applies the assembled block through a symmetric
// Gauss-Seidel sweep pair in multicolour order instead:
//
//   * the matrix: for every node row the 2x2 blocks (J_cc, J_c,mu, J_mu,c,
//     J_mu,mu) of its 3^dim neighbours, A[(k * 4 + e) * ld + n], neighbour
//     k = (dx + 1) + 3 (dy + 1) (+ 9 (dz + 1)); assembled cell by cell in
//     2^dim launches, one per cell colour (parity of the cell index in each
//     direction), so cells of one launch share no node and the rows are
//     summed in a fixed order without atomics;
//   * the sweeps: nodes coloured by the parity of their index (no two nodes
//     of one colour share a cell, so every colour updates independently);
//     forward y_n = D_n^-1 (r_n - sum_{colour(j) < colour(n)} A_nj y_j) for
//     colours 0 .. 2^dim - 1, backward z_n = y_n - D_n^-1 sum_{colour(j) >
//     colour(n)} A_nj z_j for colours 2^dim - 2 .. 0 (D_n = centre block,
//     inverted as the block-Jacobi preconditioner inverts it).
//
// FP32 copies of the matrix and of the inverted centre blocks serve the FP32
// Krylov solve.  Periodic constraints are not supported by this
// preconditioner (the set-up reports an error).
#include <string>

#include "sint_internal.h"
#include "sint_kernels.cuh"
#include "sint_launch.h"

namespace sint
{
  template <int DIM>
  struct ChStencil
  {
    static constexpr int NK  = DIM == 3 ? 27 : 9; // neighbours of a node row
    static constexpr int CTR = NK / 2;            // the node itself
  };

  // Per-point coefficients of the CH tangent (OperatorCahnHilliard):
  // M (DIM x DIM, column e = apply_M(unit e)), dM/dc grad mu (DIM),
  // dM/dgrad c (DIM x DIM), f_cc, the grains' summed velocity (ADV, DIM).
  template <int DIM, bool ADV>
  struct ChCoef
  {
    static constexpr int M = 0, MV = DIM * DIM, K = MV + DIM, FCC = K + DIM * DIM, VEL = FCC + 1;
    static constexpr int N = VEL + (ADV ? DIM : 0);
  };

  // Value and gradient at this thread's point from a cell's 2^dim nodal
  // values u[l] (l = lx + 2 ly + 4 lz), sum-factorised as eval_vg.
  template <int DIM, typename R>
  __device__ __forceinline__ void eval_local(const R *u, const QP<DIM, R> &w, R &val, R (&grad)[DIM])
  {
    if constexpr (DIM == 3)
      {
        R vx[2][2], dx[2][2];
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
#pragma unroll
          for (int ly = 0; ly < 2; ++ly)
            {
              const R u0 = u[2 * ly + 4 * lz], u1 = u[1 + 2 * ly + 4 * lz];
              vx[lz][ly] = w.wA[0] * u0 + w.wB[0] * u1;
              dx[lz][ly] = (u1 - u0) * w.ih[0];
            }
        R vxy[2], dxy[2], dyy[2];
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
          {
            vxy[lz] = w.wA[1] * vx[lz][0] + w.wB[1] * vx[lz][1];
            dxy[lz] = w.wA[1] * dx[lz][0] + w.wB[1] * dx[lz][1];
            dyy[lz] = (vx[lz][1] - vx[lz][0]) * w.ih[1];
          }
        val     = w.wA[2] * vxy[0] + w.wB[2] * vxy[1];
        grad[0] = w.wA[2] * dxy[0] + w.wB[2] * dxy[1];
        grad[1] = w.wA[2] * dyy[0] + w.wB[2] * dyy[1];
        grad[2] = (vxy[1] - vxy[0]) * w.ih[2];
      }
    else
      {
        R vx[2], dx[2];
#pragma unroll
        for (int ly = 0; ly < 2; ++ly)
          {
            const R u0 = u[2 * ly], u1 = u[1 + 2 * ly];
            vx[ly]     = w.wA[0] * u0 + w.wB[0] * u1;
            dx[ly]     = (u1 - u0) * w.ih[0];
          }
        val     = w.wA[1] * vx[0] + w.wB[1] * vx[1];
        grad[0] = w.wA[1] * dx[0] + w.wB[1] * dx[1];
        grad[1] = (vx[1] - vx[0]) * w.ih[1];
      }
  }

  // Cells of colour `colour` (bit d = parity in direction d) taken in bricks
  // of Tile<DIM> cells of the colour's coarse lattice; one thread per (cell,
  // point).  Adds each cell's element matrix of the CH block into the rows of
  // its nodes.  CUT: absent grains have zero values there (grain cut-off of
  // the preconditioner).  ADV: J_cc gains -(psi_m sum_i v_i, grad phi_l)
  // (precondition_advection_ch, operator_sintering_generic.h:800-824).
  template <int DIM, int G, bool TENS, bool CUT, bool ADV>
  __global__ void __launch_bounds__(Tile<DIM>::THREADS)
    ch_matrix_kernel(const Grid g, const Phys ph, const double *__restrict__ lin, int colour, double *__restrict__ A,
                     const uint16_t *__restrict__ mask, const AdvData adv)
  {
    using T          = Tile<DIM>;
    using CF         = ChCoef<DIM, ADV>;
    constexpr int C  = G + 2;
    constexpr int NQ = T::NQ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *s_nodes = reinterpret_cast<double *>(smem_raw); // [comp][cell][l]
    double *s_coef  = s_nodes + C * T::THREADS;              // [cell][q][coef]

    const int p[3] = {colour & 1, (colour >> 1) & 1, (colour >> 2) & 1};
    int       mc[3], ntc[3];
    const int TT[3] = {T::TX, T::TY, T::TZ};
#pragma unroll
    for (int d = 0; d < 3; ++d)
      {
        mc[d]  = d < DIM ? (g.n[d] - p[d] + 1) / 2 : 1;
        ntc[d] = (mc[d] + TT[d] - 1) / TT[d];
      }
    long long b = blockIdx.x;
    const int bx = int(b % ntc[0]);
    b /= ntc[0];
    const int by = int(b % ntc[1]);
    const int bz = int(b / ntc[1]);
    const int cell = threadIdx.x / NQ, q = threadIdx.x & (NQ - 1);
    const int lcx = cell % T::TX, lcy = (cell / T::TX) % T::TY, lcz = cell / (T::TX * T::TY);
    const int ca = bx * T::TX + lcx, cb = by * T::TY + lcy, cc = bz * T::TZ + lcz; // coarse cell coordinates
    const bool valid = ca < mc[0] && cb < mc[1] && (DIM == 2 || cc < mc[2]);
    const int  ci = 2 * ca + p[0], cj = 2 * cb + p[1], ck = DIM == 3 ? 2 * cc + p[2] : 0;
    // node q of this cell (as local node l = q for the staging)
    const long long node = valid ? node_index(g, ci + (q & 1), cj + ((q >> 1) & 1), ck + ((q >> 2) & 1)) : 0;
    for (int comp = 0; comp < C; ++comp)
      s_nodes[(comp * T::CELLS + cell) * NQ + q] = valid ? lin[comp * g.ld + node] : 0.0;
    const long long n_cells = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long lcell   = ci + (long long)g.n[0] * (cj + (long long)g.n[1] * ck);
    const unsigned  gmask   = (CUT && valid) ? mask[lcell] : ~0u;
    __syncthreads();

    const PhysR<double>   pr(ph);
    const QP<DIM, double> w(g);
    {
      double c, gc[DIM], mu_unused, gmu[DIM];
      eval_local<DIM>(s_nodes + (0 * T::CELLS + cell) * NQ, w, c, gc);
      eval_local<DIM>(s_nodes + (1 * T::CELLS + cell) * NQ, w, mu_unused, gmu);
      double eta[gdim(G)];
      double geta[gdim(G)][DIM];
#pragma unroll
      for (int i = 0; i < G; ++i)
        {
          eval_local<DIM>(s_nodes + ((2 + i) * T::CELLS + cell) * NQ, w, eta[i], geta[i]);
          if (CUT && ((gmask >> i) & 1u) == 0u)
            {
              eta[i] = 0.0;
#pragma unroll
              for (int d = 0; d < DIM; ++d)
                geta[i][d] = 0.0;
            }
        }
      double *cf = s_coef + threadIdx.x * CF::N;
      {
        double Mm[DIM][DIM];
        mobility_matrix<DIM, G, TENS>(pr, c, eta, gc, geta, Mm);
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int bb = 0; bb < DIM; ++bb)
            cf[CF::M + a * DIM + bb] = Mm[a][bb];
      }
      double mv[DIM];
      dM_dc_times<DIM, TENS>(pr, c, gc, gmu, mv);
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        cf[CF::MV + d] = mv[d];
      double Km[DIM][DIM];
      dM_dgrad_c<DIM, TENS>(pr, c, gc, gmu, Km);
#pragma unroll
      for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int bb = 0; bb < DIM; ++bb)
          cf[CF::K + a * DIM + bb] = Km[a][bb];
      const double omc = 1.0 - c;
      cf[CF::FCC] = 2.0 * pr.A * (c * c) + 4.0 * pr.A * c * (2.0 * c - 2.0) + 2.0 * pr.A * (omc * omc) + 2.0 * pr.B;
      if constexpr (ADV)
        {
          double vs[3] = {0.0, 0.0, 0.0};
          if (valid)
            {
              const double gp0 = 0.5 - 0.5 / sqrt(3.0), gp1 = 0.5 + 0.5 / sqrt(3.0);
              const int    co[3] = {ci, cj, ck};
#pragma unroll 1
              for (int i = 0; i < G; ++i)
                {
                  if (CUT && ((gmask >> i) & 1u) == 0u)
                    continue;
                  int s = adv.cell_segments[i * n_cells + lcell];
                  if (s < 0 || s >= adv.n_segments)
                    continue;
                  const double *d    = adv.segments + 9 * (long long)s;
                  double        r[3] = {0.0, 0.0, 0.0};
#pragma unroll
                  for (int e = 0; e < DIM; ++e)
                    r[e] = adv.origin[e] + (co[e] + (((q >> e) & 1) ? gp1 : gp0)) * g.h[e] - d[6 + e];
                  vs[0] += d[0] + d[4] * r[2] - d[5] * r[1];
                  vs[1] += d[1] + d[5] * r[0] - d[3] * r[2];
                  vs[2] += d[2] + d[3] * r[1] - d[4] * r[0];
                }
            }
#pragma unroll
          for (int e = 0; e < DIM; ++e)
            cf[CF::VEL + e] = vs[e];
        }
    }
    __syncthreads();
    if (!valid)
      return;

    // this thread: row of local node l = q; columns m = 0 .. NQ - 1
    const int l = q;
    // phi_a(x_q) and grad phi_a(x_q) of local node a at point qq
    auto shape = [&](int a, int qq, double &phi, double (&dphi)[DIM]) {
      phi = 1.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        phi *= (((a >> d) & 1) == ((qq >> d) & 1)) ? w.g1 : w.g0;
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        {
          double v = (((a >> d) & 1) ? 1.0 : -1.0) * w.ih[d];
#pragma unroll
          for (int e = 0; e < DIM; ++e)
            if (e != d)
              v *= (((a >> e) & 1) == ((qq >> e) & 1)) ? w.g1 : w.g0;
          dphi[d] = v;
        }
    };
    const long long row = node_index(g, ci + (l & 1), cj + ((l >> 1) & 1), ck + ((l >> 2) & 1));
#pragma unroll 1
    for (int m = 0; m < NQ; ++m)
      {
        double J[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
        for (int qq = 0; qq < NQ; ++qq)
          {
            const double *cf = s_coef + (cell * NQ + qq) * CF::N;
            double        phi, dphi[DIM], psi, dpsi[DIM];
            shape(l, qq, phi, dphi);
            shape(m, qq, psi, dpsi);
            // unknown c: flux dM/dc grad mu psi + dM/dgrad c grad psi (- v psi)
            double fl[DIM], mg[DIM];
#pragma unroll
            for (int a = 0; a < DIM; ++a)
              {
                double k = 0.0, mm = 0.0;
#pragma unroll
                for (int bb = 0; bb < DIM; ++bb)
                  {
                    k += cf[CF::K + a * DIM + bb] * dpsi[bb];
                    mm += cf[CF::M + a * DIM + bb] * dpsi[bb];
                  }
                fl[a] = cf[CF::MV + a] * psi + k;
                if constexpr (ADV)
                  fl[a] -= cf[CF::VEL + a] * psi;
                mg[a] = mm;
              }
            double gfl = 0.0, gm = 0.0, gg = 0.0;
#pragma unroll
            for (int a = 0; a < DIM; ++a)
              {
                gfl += fl[a] * dphi[a];
                gm += mg[a] * dphi[a];
                gg += dpsi[a] * dphi[a];
              }
            const double pp = psi * phi;
            J[0] += w.JxW * (pr.w0 * pp + gfl);
            J[1] += w.JxW * gm;
            J[2] += w.JxW * (-cf[CF::FCC] * pp - pr.kc * gg);
            J[3] += w.JxW * (pr.walg * pp);
          }
        const int dx = (m & 1) - (l & 1), dy = ((m >> 1) & 1) - ((l >> 1) & 1),
                  dz = DIM == 3 ? ((m >> 2) & 1) - ((l >> 2) & 1) : 0;
        const int k = (dx + 1) + 3 * (dy + 1) + (DIM == 3 ? 9 * (dz + 1) : 0);
#pragma unroll
        for (int e = 0; e < 4; ++e)
          A[(k * 4 + e) * g.ld + row] += J[e];
      }
  }

  // The nodes of colour c (bit d = parity of the index in direction d) form
  // the lattice x = 2 a + p0, y = 2 b + p1 (, z = 2 c + p2) of m[c][d] nodes
  // per direction, t = a + m0 (b + m1 c) their index in it.  The FP32 copy of
  // the matrix and of the centre-block inverses, which the FP32 Krylov solve
  // sweeps, is stored colour by colour, each colour's rows entry-major over
  // t: one colour's sweep then reads them contiguously (in node order a
  // colour's rows are every other element in x, and half of every sector read
  // would be another colour's).
  struct ColourLattice
  {
    long long cnt[8]; // nodes of the colour
    long long off[8]; // nodes of the colours before it
    int       m[8][3];
  };

  template <int DIM>
  ColourLattice colour_lattice(const Grid &g)
  {
    ColourLattice L{};
    long long     off = 0;
    for (int col = 0; col < 8; ++col)
      {
        long long cnt = col < (1 << DIM) ? 1 : 0;
        for (int d = 0; d < 3; ++d)
          {
            L.m[col][d] = d < DIM ? (g.nn[d] - ((col >> d) & 1) + 1) / 2 : 1;
            cnt *= L.m[col][d];
          }
        L.cnt[col] = cnt;
        L.off[col] = off;
        off += cnt;
      }
    return L;
  }

  // Centre-block inverses (guarded as precond_invert_kernel) in both
  // precisions and the FP32 copies of the matrix and of the inverses in the
  // colour-major layout.
  template <int DIM>
  __global__ void ch_matrix_finish_kernel(const Grid g, const ColourLattice cl, const double *__restrict__ A,
                                          float *__restrict__ A32, double *__restrict__ dinv64,
                                          float *__restrict__ dinv32)
  {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.N)
      return;
    constexpr int   NK = ChStencil<DIM>::NK, CTR = ChStencil<DIM>::CTR;
    const long long ld = g.ld;
    const int       x = int(n % g.nn[0]), y = int((n / g.nn[0]) % g.nn[1]);
    const int       z = DIM == 3 ? int(n / ((long long)g.nn[0] * g.nn[1])) : 0;
    const int       col = (x & 1) | ((y & 1) << 1) | ((z & 1) << 2);
    const long long t   = (x >> 1) + (long long)cl.m[col][0] * ((y >> 1) + (long long)cl.m[col][1] * (z >> 1));
    const long long cnt = cl.cnt[col];
    float          *a32 = A32 + cl.off[col] * (NK * 4) + t;
    for (int i = 0; i < NK * 4; ++i)
      a32[i * cnt] = float(A[i * ld + n]);
    const double a = A[(CTR * 4 + 0) * ld + n], b = A[(CTR * 4 + 1) * ld + n], c = A[(CTR * 4 + 2) * ld + n],
                 d = A[(CTR * 4 + 3) * ld + n];
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
        i00 = fabs(a) > 1.0e-10 ? 1.0 / a : 1.0;
        i11 = fabs(d) > 1.0e-10 ? 1.0 / d : 1.0;
        i01 = i10 = 0.0;
      }
    const double inv[4] = {i00, i01, i10, i11};
    for (int e = 0; e < 4; ++e)
      {
        dinv64[e * ld + n]                   = inv[e];
        dinv32[cl.off[col] * 4 + e * cnt + t] = float(inv[e]);
      }
  }

  // One colour of the forward (FWD) or backward sweep; z holds the c and mu
  // blocks of the result (y of the forward sweep, overwritten by the
  // backward one).  Neighbours are summed in the order k = 0 .. NK - 1.
  // The matrix and the inverses: node-major rows (FP64, stride ld) or the
  // colour-major FP32 copies (entry stride = the colour's node count).
  template <int DIM, typename R, bool FWD>
  __global__ void __launch_bounds__(256)
    ch_sgs_kernel(const Grid g, int colour, const ColourLattice cl, const R *__restrict__ A,
                  const R *__restrict__ dinv, const R *__restrict__ r, R *__restrict__ z)
  {
    constexpr int  NK = ChStencil<DIM>::NK;
    constexpr bool CM = sizeof(R) == 4; // colour-major matrix
    const int      p[3] = {colour & 1, (colour >> 1) & 1, (colour >> 2) & 1};
    const int      m0 = cl.m[colour][0], m1 = cl.m[colour][1];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cl.cnt[colour])
      return;
    const int a = int(t % m0), b = int((t / m0) % m1), c = int(t / ((long long)m0 * m1));
    const int x = 2 * a + p[0], y = 2 * b + p[1], zz = DIM == 3 ? 2 * c + p[2] : 0;
    const long long n  = node_index(g, x, y, zz);
    const long long ld = g.ld;
    // row entries of this node: A_row[i * as]
    const long long as    = CM ? cl.cnt[colour] : ld;
    const R        *A_row = CM ? A + cl.off[colour] * (NK * 4) + t : A + n;
    const R        *d_row = CM ? dinv + cl.off[colour] * 4 + t : dinv + n;
    R               s0 = R(0), s1 = R(0);
#pragma unroll
    for (int k = 0; k < NK; ++k)
      {
        const int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = DIM == 3 ? k / 9 - 1 : 0;
        // the neighbour's colour: odd offsets flip the parity
        const int nc = colour ^ ((dx & 1) | ((dy & 1) << 1) | ((dz & 1) << 2));
        if (FWD ? !(nc < colour) : !(nc > colour))
          continue;
        const int xx = x + dx, yy = y + dy, zn = zz + dz;
        if (xx < 0 || yy < 0 || zn < 0 || xx >= g.nn[0] || yy >= g.nn[1] || zn >= g.nn[2])
          continue;
        const long long j  = node_index(g, xx, yy, zn);
        const R         v0 = z[j], v1 = z[ld + j];
        s0 += A_row[(k * 4 + 0) * as] * v0 + A_row[(k * 4 + 1) * as] * v1;
        s1 += A_row[(k * 4 + 2) * as] * v0 + A_row[(k * 4 + 3) * as] * v1;
      }
    const R i00 = d_row[0], i01 = d_row[as], i10 = d_row[2 * as], i11 = d_row[3 * as];
    if (FWD)
      {
        const R a0 = r[n] - s0, a1 = r[ld + n] - s1;
        z[n]       = i00 * a0 + i01 * a1;
        z[ld + n]  = i10 * a0 + i11 * a1;
      }
    else
      {
        z[n]      = z[n] - (i00 * s0 + i01 * s1);
        z[ld + n] = z[ld + n] - (i10 * s0 + i11 * s1);
      }
  }

  template <int DIM, int G, bool TENS, bool CUT, bool ADV>
  static cudaError_t launch_ch_matrix_g(const Grid &g, const Ctx *c, int colour, long long blocks, size_t smem,
                                        const uint16_t *mask, const AdvData &adv, cudaStream_t s)
  {
    auto k = ch_matrix_kernel<DIM, G, TENS, CUT, ADV>;
    if (smem > 48 * 1024)
      if (cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)))
        return e;
    k<<<dim3((unsigned)blocks), Tile<DIM>::THREADS, smem, s>>>(g, c->phys, c->lin64, colour, c->ch_A64, mask, adv);
    count_launches(1);
    return cudaGetLastError();
  }

  template <int DIM, bool TENS, bool CUT, bool ADV>
  static cudaError_t launch_ch_matrix(int G, const Grid &g, const Ctx *c, int colour, long long blocks, size_t smem,
                                      const uint16_t *mask, const AdvData &adv, cudaStream_t s)
  {
    switch (G)
      {
#define SINT_CASE(GG)                                                                                             \
  case GG: return launch_ch_matrix_g<DIM, GG, TENS, CUT, ADV>(g, c, colour, blocks, smem, mask, adv, s);
        SINT_CASE(1) SINT_CASE(2) SINT_CASE(3) SINT_CASE(4) SINT_CASE(5) SINT_CASE(6)
        SINT_CASE(7) SINT_CASE(8) SINT_CASE(9) SINT_CASE(10) SINT_CASE(11) SINT_CASE(12)
#undef SINT_CASE
      }
    return cudaErrorInvalidValue;
  }

  template <int DIM, bool TENS, bool CUT, bool ADV>
  static cudaError_t assemble_dim(const Ctx *c, const uint16_t *mask, const AdvData &adv, cudaStream_t s)
  {
    using T           = Tile<DIM>;
    const int    G    = c->G;
    const size_t smem = (size_t(G + 2) * T::THREADS + size_t(ChCoef<DIM, ADV>::N) * T::THREADS) * sizeof(double);
    const Grid  &g    = c->grid;
    for (int colour = 0; colour < (1 << DIM); ++colour)
      {
        long long blocks = 1;
        const int TT[3]  = {T::TX, T::TY, T::TZ};
        for (int d = 0; d < DIM; ++d)
          {
            const int m = (g.n[d] - ((colour >> d) & 1) + 1) / 2;
            blocks *= (m + TT[d] - 1) / TT[d];
          }
        if (blocks == 0)
          continue;
        const cudaError_t e = launch_ch_matrix<DIM, TENS, CUT, ADV>(G, g, c, colour, blocks, smem, mask, adv, s);
        if (e != cudaSuccess)
          return e;
      }
    const long long nb = (c->N + 255) / 256;
    ch_matrix_finish_kernel<DIM><<<dim3((unsigned)nb), 256, 0, s>>>(g, colour_lattice<DIM>(g), c->ch_A64, c->ch_A32,
                                                                   c->ch_dinv64, c->ch_dinv32);
    count_launches(1);
    return cudaGetLastError();
  }

  template <int DIM>
  static cudaError_t assemble_mob(const Ctx *c, cudaStream_t s)
  {
    const uint16_t *m   = preconditioner_mask(c);
    const AdvData  *adv = active_adv(c);
    const bool      t   = c->params.tensorial != 0;
#define SINT_ASM(TT, CC, AA) assemble_dim<DIM, TT, CC, AA>(c, m, adv ? *adv : AdvData(), s)
    if (t)
      return m ? (adv ? SINT_ASM(true, true, true) : SINT_ASM(true, true, false))
               : (adv ? SINT_ASM(true, false, true) : SINT_ASM(true, false, false));
    return m ? (adv ? SINT_ASM(false, true, true) : SINT_ASM(false, true, false))
             : (adv ? SINT_ASM(false, false, true) : SINT_ASM(false, false, false));
#undef SINT_ASM
  }

  int ch_sgs_setup(Ctx *c, cudaStream_t s)
  {
    if (c->grid.periodic)
      {
        set_error("sint_precond_setup: the Cahn-Hilliard Gauss-Seidel preconditioner does not support periodic "
                  "constraints; use the block-Jacobi preconditioner");
        return SINT_ERR_ARG;
      }
    const int    NK  = c->grid.dim == 3 ? ChStencil<3>::NK : ChStencil<2>::NK;
    const size_t mat = size_t(NK) * 4 * size_t(c->ld);
    cudaError_t  e   = cudaSuccess;
    if (!c->ch_A64)
      {
        if ((e = cudaMalloc(&c->ch_A64, mat * sizeof(double))) != cudaSuccess ||
            (e = cudaMalloc(&c->ch_A32, mat * sizeof(float))) != cudaSuccess ||
            (e = cudaMalloc(&c->ch_dinv64, 4 * size_t(c->ld) * sizeof(double))) != cudaSuccess ||
            (e = cudaMalloc(&c->ch_dinv32, 4 * size_t(c->ld) * sizeof(float))) != cudaSuccess)
          return cuda_fail(e, "sint_precond_setup: Cahn-Hilliard matrix allocation");
        // padding rows stay zero
        if ((e = cudaMemset(c->ch_dinv64, 0, 4 * size_t(c->ld) * sizeof(double))) != cudaSuccess ||
            (e = cudaMemset(c->ch_dinv32, 0, 4 * size_t(c->ld) * sizeof(float))) != cudaSuccess ||
            (e = cudaMemset(c->ch_A32, 0, mat * sizeof(float))) != cudaSuccess)
          return cuda_fail(e, "sint_precond_setup: Cahn-Hilliard matrix clear");
      }
    if ((e = cudaMemsetAsync(c->ch_A64, 0, mat * sizeof(double), s)) != cudaSuccess)
      return cuda_fail(e, "sint_precond_setup: Cahn-Hilliard matrix clear");
    e = c->grid.dim == 3 ? assemble_mob<3>(c, s) : assemble_mob<2>(c, s);
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_precond_setup: Cahn-Hilliard matrix");
  }

  template <int DIM, typename R>
  static cudaError_t sweeps(const Grid &g, const R *A, const R *dinv, const R *r, R *z, cudaStream_t s)
  {
    constexpr int       NCOL = 1 << DIM;
    const ColourLattice cl   = colour_lattice<DIM>(g);
    auto                launch = [&](int colour, bool fwd) -> cudaError_t {
      const long long cnt = cl.cnt[colour];
      if (cnt == 0)
        return cudaSuccess;
      const unsigned nb = (unsigned)((cnt + 255) / 256);
      if (fwd)
        ch_sgs_kernel<DIM, R, true><<<nb, 256, 0, s>>>(g, colour, cl, A, dinv, r, z);
      else
        ch_sgs_kernel<DIM, R, false><<<nb, 256, 0, s>>>(g, colour, cl, A, dinv, r, z);
      count_launches(1);
      return cudaGetLastError();
    };
    for (int col = 0; col < NCOL; ++col)
      if (cudaError_t e = launch(col, true))
        return e;
    for (int col = NCOL - 2; col >= 0; --col)
      if (cudaError_t e = launch(col, false))
        return e;
    return cudaSuccess;
  }

  template <typename R>
  cudaError_t ch_sgs_apply(const Ctx *c, const R *r, R *z, cudaStream_t s)
  {
    const R *A    = sizeof(R) == 8 ? reinterpret_cast<const R *>(c->ch_A64) : reinterpret_cast<const R *>(c->ch_A32);
    const R *dinv = sizeof(R) == 8 ? reinterpret_cast<const R *>(c->ch_dinv64)
                                   : reinterpret_cast<const R *>(c->ch_dinv32);
    return c->grid.dim == 3 ? sweeps<3, R>(c->grid, A, dinv, r, z, s) : sweeps<2, R>(c->grid, A, dinv, r, z, s);
  }
  template cudaError_t ch_sgs_apply<double>(const Ctx *, const double *, double *, cudaStream_t);
  template cudaError_t ch_sgs_apply<float>(const Ctx *, const float *, float *, cudaStream_t);
} // namespace sint
