// Shared device-side building blocks of the sintering cell kernels.
//
// Mesh: uniform Cartesian Q1 cells, nodes numbered lexicographically
// (x fastest).  A thread block owns a brick ("tile") of cells; one thread
// per (cell, quadrature point), so the 2^dim threads of a cell sit in
// consecutive lanes and exchange data with warp shuffles.
//
// Data flow of a cell kernel
//   1. the tile's node box (TX+1)(TY+1)(TZ+1) of every input component is
//      staged in shared memory with coalesced loads;
//   2. each thread evaluates values and gradients at its quadrature point by
//      sum factorisation over the cell's 2^dim nodal values (1D Q1 matrices
//      at the two Gauss points are 2x2);
//   3. the point-wise physics (free energy, mobility) runs in registers;
//   4. integration (test functions) is a sum-factorised butterfly across the
//      2^dim lanes of a cell: afterwards lane l holds the cell's contribution
//      to its local node l;
//   5. the contributions are summed per node inside the tile in a fixed order
//      (no atomics); nodes whose every adjacent cell lies in the tile are
//      written to the output, nodes on a tile face go to a per-tile partial
//      buffer that a second kernel (combine) sums in a fixed order.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "sint_f2.cuh"

namespace sint
{
  constexpr int MAX_GRAINS = 12;

  template <int DIM>
  struct Tile;

  template <>
  struct Tile<3>
  {
    static constexpr int TX = 4, TY = 4, TZ = 2;
    static constexpr int NQ      = 8;
    static constexpr int CELLS   = TX * TY * TZ;
    static constexpr int BX      = TX + 1, BY = TY + 1, BZ = TZ + 1;
    static constexpr int BOX     = BX * BY * BZ;
    // storage of a node box in shared memory: node (bx, by, bz) at
    // bx + SY by + SZ bz.  With these pitches the base nodes of a warp's 32
    // cells (4 x 4 x 2) fall on every 8-byte bank pair exactly twice (FP64:
    // two wavefronts, the minimum) and on 32 distinct 4-byte banks (FP32)
    static constexpr int SY = 8, SZ = 44;
    static constexpr int BOXS    = (BX - 1) + SY * (BY - 1) + SZ * (BZ - 1) + 1;
    static constexpr int THREADS = CELLS * NQ;
    // node contributions are parked as [comp][l][cell] with row pitch CP: the
    // +2 makes both the write (lane = cell * 8 + l) and the per-node read
    // (consecutive cells) free of shared-memory bank conflicts
    static constexpr int CP = CELLS + 2;
    static constexpr int CS = NQ * CP; // per component
    static constexpr int NG = THREADS / BOX; // node-major phases: threads per box node
  };

  template <>
  struct Tile<2>
  {
    static constexpr int TX = 8, TY = 8, TZ = 1;
    static constexpr int NQ      = 4;
    static constexpr int CELLS   = TX * TY;
    static constexpr int BX      = TX + 1, BY = TY + 1, BZ = 1;
    static constexpr int BOX     = BX * BY;
    static constexpr int SY = BX, SZ = BOX; // dense storage
    static constexpr int BOXS    = BOX;
    static constexpr int THREADS = CELLS * NQ;
    static constexpr int CP      = CELLS + 4;
    static constexpr int CS      = NQ * CP;
    static constexpr int NG      = THREADS / BOX;
  };

  // Mesh description passed by value to every kernel.
  struct Grid
  {
    int       dim;
    int       n[3];  // cells per direction (1 for unused directions)
    int       nn[3]; // nodes per direction (1 for unused directions)
    int       nt[3]; // tiles per direction (1 for unused directions)
    long long N;     // number of nodes
    long long ld;    // block stride of a DoF vector
    long long n_tiles;
    double    h[3];
    // Exact element Laplacian of the uniform cell, K_lm = kx[l xor m]
    // (kx[x] = int grad phi_l . grad phi_(l xor x)), in both precisions.
    double kxd[8];
    float  kxf[8];
    // The same stencil times the coefficient of each constant-coefficient
    // gradient row: kst[0] = -kappa_c kx (mu row, acting on c), kst[1] =
    // L kappa_p kx (eta rows); refreshed by set_row_stiffness whenever
    // kappa_c, kappa_p or L change.
    double kstd[2][8];
    float  kstf[2][8];
    // division by nt[0] and nt[1] as multiply-shift (exact for n < 2^31):
    // n / nt[d] = (n * mdiv[d]) >> (32 + sdiv[d])
    unsigned long long mdiv[2];
    int                sdiv[2];
    // the same for nn[0] and nn[1] (node index -> node coordinates; N < 2^31)
    unsigned long long mnode[2];
    int                snode[2];
    // periodic directions (bit d): the nodes at coordinate n[d] are constrained
    // to the nodes at 0 (DoFTools::make_periodicity_constraints), so the cell
    // kernels read the master values there
    int periodic = 0;
  };

  // Granlund-Montgomery division by an invariant integer d >= 1: with
  // s = ceil(log2 d) and m = ceil(2^(32+s) / d), floor(n / d) = (n m) >> (32+s)
  // for every 0 <= n < 2^31 (m < 2^33, so n m < 2^64).
  inline void make_divisor(unsigned d, unsigned long long &m, int &s)
  {
    s = 0;
    while ((1ull << s) < d)
      ++s;
    const unsigned long long num = 1ull << (32 + s);
    m                            = num / d + (num % d != 0 ? 1 : 0);
  }

  __device__ __forceinline__ unsigned fast_div(unsigned n, unsigned long long m, int s)
  {
    return (unsigned)(((unsigned long long)n * m) >> (32 + s));
  }

  // Row coefficients of the element Laplacian (Grid::kstd / kstf).
  inline void set_row_stiffness(Grid &g, double kappa_c, double kappa_p, double L)
  {
    for (int x = 0; x < 8; ++x)
      {
        g.kstd[0][x] = -kappa_c * g.kxd[x];
        g.kstd[1][x] = L * kappa_p * g.kxd[x];
        g.kstf[0][x] = float(g.kstd[0][x]);
        g.kstf[1][x] = float(g.kstd[1][x]);
      }
  }

  template <typename R>
  __device__ __forceinline__ R kst(const Grid &g, int row, int x);
  template <>
  __device__ __forceinline__ double kst<double>(const Grid &g, int row, int x)
  {
    return g.kstd[row][x];
  }
  template <>
  __device__ __forceinline__ float kst<float>(const Grid &g, int row, int x)
  {
    return g.kstf[row][x];
  }
  template <>
  __device__ __forceinline__ F2 kst<F2>(const Grid &g, int row, int x)
  {
    return F2(g.kstf[row][x]);
  }

  template <typename R>
  __device__ __forceinline__ R kx(const Grid &g, int x);
  template <>
  __device__ __forceinline__ double kx<double>(const Grid &g, int x)
  {
    return g.kxd[x];
  }
  template <>
  __device__ __forceinline__ float kx<float>(const Grid &g, int x)
  {
    return g.kxf[x];
  }
  template <>
  __device__ __forceinline__ F2 kx<F2>(const Grid &g, int x)
  {
    return F2(g.kxf[x]);
  }

  // Device form of the residual's range hooks (pre_operation /
  // post_operation of evaluate_nonlinear_residual,
  // operator_sintering_generic.h:393-401), as the Jacobian-free operator uses
  // them (lac/jacobian_operator.h:160-232): the residual is evaluated at
  // src + perturb_scale * perturb (formed while the node boxes are staged, src
  // is never modified), and with `epilogue` the result is stored as
  // (R - subtract) * scale (fused into the stores and the combine step).
  struct ResidualHooks
  {
    const double *perturb       = nullptr;
    double        perturb_scale = 0.0;
    const double *subtract      = nullptr; // may be null: (R - 0) * scale
    double        scale         = 1.0;
    int           epilogue      = 0;
  };

  // Point-wise model parameters (FP64 on the host, cast per kernel), and the
  // residual hooks of one evaluation (left empty everywhere else).
  struct Phys
  {
    double A, B, kappa_c, kappa_p;
    double Mvol, Mvap, Msurf, Mgb, L;
    double w0, w_alg;
    double w_hist[4];
    int    order;
    ResidualHooks hooks;
  };

  template <typename R>
  struct PhysR
  {
    R A, B, kc, kp, Mvol, Mvap, Msurf, Mgb, L, w0, walg;
    __host__ __device__ PhysR() {}
    __host__ __device__ explicit PhysR(const Phys &p)
      : A(R(p.A)), B(R(p.B)), kc(R(p.kappa_c)), kp(R(p.kappa_p)), Mvol(R(p.Mvol)), Mvap(R(p.Mvap)),
        Msurf(R(p.Msurf)), Mgb(R(p.Mgb)), L(R(p.L)), w0(R(p.w0)), walg(R(p.w_alg))
    {}
  };

  // Tile coordinates of this block.
  struct TileCoord
  {
    int       t[3];   // tile index per direction
    int       o[3];   // first cell of the tile per direction
    long long linear; // blockIdx.x
  };

  // Grain cut-off, as the kernels see it.  Tiles are sorted into classes by
  // the number of grains relevant on any of their cells: class k's tiles are
  // tiles[range[k] .. range[k + 1]), and the kernel instantiated for k grains
  // works on the compacted components (c, mu, eta_{l_0}, .., eta_{l_(k-1)})
  // with the tile's grain list l packed four bits per grain in
  // tile_grains[tile] -- the src_view of do_vmult_range_no_template
  // (operator_sintering_generic.h:496-509) per tile instead of per cell batch.
  // The arrays below `tiles` are in the sorted order of `tiles`.
  struct CutTiles
  {
    const uint16_t           *cell_mask   = nullptr; // per cell: bit b = grain b relevant
    const int                *tiles       = nullptr; // tile ids sorted by class
    const unsigned long long *tile_grains = nullptr; // the tile's packed grain list
    const uint16_t           *tile_mask   = nullptr; // the union of the tile's cell masks
    const int                *range       = nullptr; // class offsets into tiles (n_grains + 2)
    int                       c_all       = 0;       // components of the full operator
  };

  // Advection (rigid-body motion of the grains), as the kernels see it:
  // cell_segments[b * n_cells + cell] = segment of order parameter b the cell
  // belongs to (-1: none; ids >= n_segments count as none); segments[9 s ..]
  // = translational velocity (3), angular velocity (3; z only in 2D) and
  // center (3) of segment s.  Grain b moves with v_t + w x (x - center) on
  // the cells of its segment (AdvectionVelocityData::get_velocity,
  // sintering/advection.h:247-263).
  struct AdvData
  {
    const int    *cell_segments = nullptr;
    const double *segments      = nullptr;
    int           n_segments    = 0;
    int           reserved      = 0; // explicit padding: the struct is compared bytewise
    double        origin[3]     = {0.0, 0.0, 0.0};
  };

  // Size of a per-grain array: at least one element (the grain cut-off runs
  // tiles without any relevant grain through the G = 0 kernels).
  __host__ __device__ constexpr int gdim(int G) { return G > 0 ? G : 1; }

  // Component of the full vector behind compacted component b.
  __device__ __forceinline__ int comp_of(int b, unsigned long long gl)
  {
    return b < 2 ? b : 2 + int((gl >> (4 * (b - 2))) & 15ull);
  }

  template <int DIM>
  __device__ __forceinline__ TileCoord tile_coord(const Grid &g)
  {
    using T = Tile<DIM>;
    TileCoord tc;
    tc.linear    = blockIdx.x;
    long long r  = tc.linear;
    tc.t[0]      = int(r % g.nt[0]);
    r /= g.nt[0];
    tc.t[1] = int(r % g.nt[1]);
    r /= g.nt[1];
    tc.t[2] = int(r);
    tc.o[0] = tc.t[0] * T::TX;
    tc.o[1] = tc.t[1] * T::TY;
    tc.o[2] = tc.t[2] * T::TZ;
    return tc;
  }

  __device__ __forceinline__ long long node_index(const Grid &g, int i, int j, int k)
  {
    return (long long)i + (long long)g.nn[0] * ((long long)j + (long long)g.nn[1] * k);
  }

  // Node-major view of the tile's node box for the load and store phases:
  // thread t serves box node t % BOX and every NG-th component starting at
  // t / BOX (threads with t / BOX >= NG idle), so the index arithmetic is done
  // once per node.
  template <int DIM>
  struct BoxNode
  {
    int       b;      // box node index
    int       sb;     // its place in the shared-memory box (pitches SY, SZ)
    int       grp;    // first component served
    int       bx, by, bz;
    bool      active; // thread serves a node
    bool      inside; // node exists in the mesh
    long long gidx;   // global node index (valid if inside): where results go
    long long lidx;   // node whose values are read: gidx, or its periodic master

    __device__ __forceinline__ BoxNode(const Grid &g, const TileCoord &tc)
    {
      using T = Tile<DIM>;
      b       = threadIdx.x % T::BOX;
      grp     = threadIdx.x / T::BOX;
      active  = grp < T::NG;
      bx      = b % T::BX;
      by      = (b / T::BX) % T::BY;
      bz      = b / (T::BX * T::BY);
      sb      = bx + T::SY * by + T::SZ * bz;
      const int gi = tc.o[0] + bx, gj = tc.o[1] + by, gk = (DIM == 3) ? tc.o[2] + bz : 0;
      inside       = gi < g.nn[0] && gj < g.nn[1] && gk < g.nn[2];
      gidx         = inside ? node_index(g, gi, gj, gk) : 0;
      lidx         = gidx;
      if (g.periodic && inside)
        lidx = node_index(g, ((g.periodic & 1) && gi == g.n[0]) ? 0 : gi, ((g.periodic & 2) && gj == g.n[1]) ? 0 : gj,
                          ((g.periodic & 4) && gk == g.n[2]) ? 0 : gk);
    }
  };

  // The same node-major view, fixed for a whole launch: computed once per
  // thread, it serves every tile.  For an interior tile (one that touches no
  // mesh boundary: o[d] > 0 and o[d] + T[d] < n[d]) every box node exists,
  // none is a periodic slave, and a node is owned by the tile exactly when it
  // lies on no face of the box, so the load and the store need only the
  // tile's first node plus the thread's fixed offset.
  template <int DIM>
  struct NodePlan
  {
    int      b, grp; // box node, first component served
    int      sb;     // its place in the shared-memory box
    bool     active;
    bool     inner;  // on no face of the box (owned in an interior tile)
    int      off;    // node offset from the tile's first node: bx + nn0 (by + nn1 bz)
    unsigned ok;     // bit l: the cell whose local node l this is lies in the tile
    int      cbase;  // contribution offset of local node 0: bx + TX (by + TY bz)

    __device__ __forceinline__ explicit NodePlan(const Grid &g)
    {
      using T = Tile<DIM>;
      b       = threadIdx.x % T::BOX;
      grp     = threadIdx.x / T::BOX;
      active  = grp < T::NG;
      const int bx = b % T::BX, by = (b / T::BX) % T::BY, bz = b / (T::BX * T::BY);
      sb           = bx + T::SY * by + T::SZ * bz;
      inner        = bx > 0 && bx < T::TX && by > 0 && by < T::TY && (DIM == 2 || (bz > 0 && bz < T::TZ));
      off          = bx + g.nn[0] * (by + g.nn[1] * bz);
      cbase        = bx + T::TX * (by + T::TY * bz);
      ok           = 0u;
#pragma unroll
      for (int l = 0; l < T::NQ; ++l)
        {
          const int cx = bx - (l & 1), cy = by - ((l >> 1) & 1), cz = (DIM == 3) ? bz - ((l >> 2) & 1) : 0;
          if (cx >= 0 && cx < T::TX && cy >= 0 && cy < T::TY && cz >= 0 && cz < T::TZ)
            ok |= 1u << l;
        }
    }
  };

  // Whether tile tc touches no mesh boundary (the fast path of NodePlan).
  template <int DIM>
  __device__ __forceinline__ bool tile_interior(const Grid &g, const TileCoord &tc)
  {
    using T = Tile<DIM>;
    return tc.o[0] > 0 && tc.o[0] + T::TX < g.n[0] && tc.o[1] > 0 && tc.o[1] + T::TY < g.n[1] &&
           (DIM == 2 || (tc.o[2] > 0 && tc.o[2] + T::TZ < g.n[2]));
  }

  // Global index of the first node of tile tc.
  __device__ __forceinline__ long long tile_node0(const Grid &g, const TileCoord &tc)
  {
    return node_index(g, tc.o[0], tc.o[1], tc.o[2]);
  }

  // Stage the node box of `ncomp` components of `src` (block stride g.ld) in
  // shared memory, layout s[comp * BOXS + sb]; nodes outside the mesh
  // read as zero.
  // With `mapped`, box component b is component comp_of(b, gl) of src.
  template <int DIM, typename R, typename S>
  __device__ __forceinline__ void load_box(R *s, const S *__restrict__ src, int ncomp, const Grid &g,
                                           const BoxNode<DIM> &bn, unsigned long long gl = 0, bool mapped = false,
                                           const S *__restrict__ perturb = nullptr, S perturb_scale = S(0))
  {
    using T = Tile<DIM>;
    if (!bn.active)
      return;
    const S *p = src + bn.lidx;
    for (int comp = bn.grp; comp < ncomp; comp += T::NG)
      {
        R v = R(0);
        if (bn.inside)
          {
            const long long off = (mapped ? comp_of(comp, gl) : comp) * g.ld;
            v                   = R(p[off]);
            if (perturb) // the residual's perturbation hook: src + a x
              v = R(p[off] + perturb_scale * perturb[bn.lidx + off]);
          }
        s[comp * T::BOXS + bn.sb] = v;
      }
  }

  // Asynchronous global->shared copies (cp.async, sm_80+): the node box of the
  // next tile is fetched while the current one is computed.  Nodes outside
  // the mesh are zero-filled (source size 0; the source address then only has
  // to be a valid pointer, the vector base is used).
  __device__ __forceinline__ void cp_async_elem(double *s, const double *gptr, bool valid)
  {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gptr), "r"(valid ? 8 : 0));
  }
  __device__ __forceinline__ void cp_async_elem(float *s, const float *gptr, bool valid)
  {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gptr), "r"(valid ? 4 : 0));
  }
  __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
  template <int N>
  __device__ __forceinline__ void cp_async_wait()
  {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
  }

  // Issue the asynchronous load of `ncomp` components of `src` into the box
  // buffer s (layout s[(comp * BOXS + sb) * LS]: LS = 2 fills one lane of a
  // box of packed pairs, s pointing at that lane).
  template <int DIM, typename R, int LS = 1>
  __device__ __forceinline__ void load_box_async(R *s, const R *__restrict__ src, int ncomp, const Grid &g,
                                                 const BoxNode<DIM> &bn, unsigned long long gl = 0,
                                                 bool mapped = false)
  {
    using T = Tile<DIM>;
    if (!bn.active)
      return;
    const R *p = bn.inside ? src + bn.lidx : src;
    for (int comp = bn.grp; comp < ncomp; comp += T::NG)
      cp_async_elem(s + (comp * T::BOXS + bn.sb) * LS,
                    bn.inside ? p + (mapped ? comp_of(comp, gl) : comp) * g.ld : src, bn.inside);
  }

  // Interior-tile form of load_box_async: every box node exists and is read
  // at node0 + the thread's fixed offset.
  template <int DIM, typename R, int LS = 1>
  __device__ __forceinline__ void load_box_async_interior(R *s, const R *__restrict__ src, int ncomp, const Grid &g,
                                                          const NodePlan<DIM> &np, long long node0,
                                                          unsigned long long gl = 0, bool mapped = false)
  {
    using T = Tile<DIM>;
    if (!np.active)
      return;
    const R *p = src + node0 + np.off;
    for (int comp = np.grp; comp < ncomp; comp += T::NG)
      cp_async_elem(s + (comp * T::BOXS + np.sb) * LS, p + (mapped ? comp_of(comp, gl) : comp) * g.ld, true);
  }

  template <int DIM>
  __device__ __forceinline__ TileCoord tile_coord_of(const Grid &g, long long tile)
  {
    using T = Tile<DIM>;
    TileCoord      tc;
    tc.linear         = tile;
    const unsigned n  = (unsigned)tile; // n_tiles < 2^31 (checked at set-up)
    const unsigned q0 = fast_div(n, g.mdiv[0], g.sdiv[0]);
    const unsigned q1 = fast_div(q0, g.mdiv[1], g.sdiv[1]);
    tc.t[0]           = int(n - q0 * (unsigned)g.nt[0]);
    tc.t[1]           = int(q0 - q1 * (unsigned)g.nt[1]);
    tc.t[2]           = int(q1);
    tc.o[0] = tc.t[0] * T::TX;
    tc.o[1] = tc.t[1] * T::TY;
    tc.o[2] = tc.t[2] * T::TZ;
    return tc;
  }

  // Per-thread quadrature constants.  Lane bits of (threadIdx.x % NQ) are the
  // quadrature point coordinates (qx, qy, qz); after the integration butterfly
  // they are the local node coordinates (lx, ly, lz).
  template <int DIM, typename R>
  struct QP
  {
    R wA[DIM], wB[DIM]; // interpolation weights of the two nodes at this point
    R ih[DIM];          // 1 / h
    R sgn_ih[DIM];      // (+-1) / h: derivative sign of this lane's node
    R g1, g0;           // Q1 shape values at the Gauss points: phi_l(x_q) = (l == q) ? g1 : g0
    R JxW;
    int q;
    // box offsets of the nodes l xor x of this lane's node l (stiffness stencil)
    int koff[1 << DIM];

    __device__ __forceinline__ explicit QP(const Grid &g)
    {
      q                 = threadIdx.x & ((1 << DIM) - 1);
      const double s3   = 0.5 / 1.7320508075688772935274463415058723669428; // 1 / (2 sqrt 3)
      const double gg0  = 0.5 - s3, gg1 = 0.5 + s3;
      g1                = R(gg1);
      g0                = R(gg0);
      double jxw        = 1.0;
      for (int d = 0; d < DIM; ++d)
        {
          const int b = (q >> d) & 1;
          // node 0 of the 1D element has phi_0(x_q) = 1 - x_q, node 1 has x_q
          wA[d]     = R(b ? gg0 : gg1);
          wB[d]     = R(b ? gg1 : gg0);
          ih[d]     = R(1.0 / g.h[d]);
          sgn_ih[d] = R((b ? 1.0 : -1.0) / g.h[d]);
          jxw *= 0.5 * g.h[d];
        }
      JxW = R(jxw);
      using T = Tile<DIM>;
      const int stride[3] = {1, T::SY, T::SZ};
#pragma unroll
      for (int x = 0; x < (1 << DIM); ++x)
        {
          int off = 0;
#pragma unroll
          for (int d = 0; d < DIM; ++d)
            off += (((q >> d) & 1) ^ ((x >> d) & 1)) * stride[d]; // bit d of node l xor x
          koff[x] = off;
        }
    }
  };

  // Box offset of local node (0,0,0) of cell `cell` of the tile.
  template <int DIM>
  __device__ __forceinline__ int cell_box_base(int cell)
  {
    using T      = Tile<DIM>;
    const int cx = cell % T::TX, cy = (cell / T::TX) % T::TY, cz = cell / (T::TX * T::TY);
    return cx + T::SY * cy + T::SZ * cz;
  }

  template <int DIM>
  __device__ __forceinline__ bool cell_in_mesh(int cell, const TileCoord &tc, const Grid &g)
  {
    using T      = Tile<DIM>;
    const int cx = cell % T::TX, cy = (cell / T::TX) % T::TY, cz = cell / (T::TX * T::TY);
    return tc.o[0] + cx < g.n[0] && tc.o[1] + cy < g.n[1] && (DIM == 2 || tc.o[2] + cz < g.n[2]);
  }

  // Value and gradient of one component at this thread's quadrature point,
  // by sum factorisation over the cell's nodal values in the staged box.
  template <int DIM, typename R>
  __device__ __forceinline__ void eval_vg(const R *s, int b0, const QP<DIM, R> &w, R &val, R (&grad)[DIM])
  {
    using T = Tile<DIM>;
    if constexpr (DIM == 3)
      {
        constexpr int SY = T::SY, SZ = T::SZ;
        R vx[2][2], dx[2][2];
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
#pragma unroll
          for (int ly = 0; ly < 2; ++ly)
            {
              const R u0 = s[b0 + ly * SY + lz * SZ], u1 = s[b0 + 1 + ly * SY + lz * SZ];
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
        constexpr int SY = T::SY;
        R vx[2], dx[2];
#pragma unroll
        for (int ly = 0; ly < 2; ++ly)
          {
            const R u0 = s[b0 + ly * SY], u1 = s[b0 + 1 + ly * SY];
            vx[ly]     = w.wA[0] * u0 + w.wB[0] * u1;
            dx[ly]     = (u1 - u0) * w.ih[0];
          }
        val     = w.wA[1] * vx[0] + w.wB[1] * vx[1];
        grad[0] = w.wA[1] * dx[0] + w.wB[1] * dx[1];
        grad[1] = (vx[1] - vx[0]) * w.ih[1];
      }
  }

  // Value only.
  template <int DIM, typename R>
  __device__ __forceinline__ R eval_v(const R *s, int b0, const QP<DIM, R> &w)
  {
    using T = Tile<DIM>;
    if constexpr (DIM == 3)
      {
        constexpr int SY = T::SY, SZ = T::SZ;
        R vxy[2];
#pragma unroll
        for (int lz = 0; lz < 2; ++lz)
          {
            const R a = w.wA[0] * s[b0 + lz * SZ] + w.wB[0] * s[b0 + 1 + lz * SZ];
            const R b = w.wA[0] * s[b0 + SY + lz * SZ] + w.wB[0] * s[b0 + 1 + SY + lz * SZ];
            vxy[lz]   = w.wA[1] * a + w.wB[1] * b;
          }
        return w.wA[2] * vxy[0] + w.wB[2] * vxy[1];
      }
    else
      {
        constexpr int SY = T::SY;
        const R a = w.wA[0] * s[b0] + w.wB[0] * s[b0 + 1];
        const R b = w.wA[0] * s[b0 + SY] + w.wB[0] * s[b0 + 1 + SY];
        return w.wA[1] * a + w.wB[1] * b;
      }
  }

  // Integration butterfly.  Input: this lane's point value v and gradient g
  // of a residual row at its quadrature point.  Output: the cell integral
  //   sum_q JxW (v_q phi_l(x_q) + g_q . grad phi_l(x_q))
  // for the local node l given by this lane's bits.  Sum factorised: one
  // stage per direction, each exchanging with the lane that differs in that bit.
  template <int DIM, typename R>
  __device__ __forceinline__ R integrate_butterfly(R v, const R (&g)[DIM], const QP<DIM, R> &w)
  {
    constexpr unsigned FULL = 0xffffffffu;
    if constexpr (DIM == 3)
      {
        // stage x
        const R vp = __shfl_xor_sync(FULL, v, 1), gxp = __shfl_xor_sync(FULL, g[0], 1);
        const R gyp = __shfl_xor_sync(FULL, g[1], 1), gzp = __shfl_xor_sync(FULL, g[2], 1);
        const R t   = w.g1 * v + w.g0 * vp + w.sgn_ih[0] * (g[0] + gxp);
        const R gy  = w.g1 * g[1] + w.g0 * gyp;
        const R gz  = w.g1 * g[2] + w.g0 * gzp;
        // stage y
        const R tp = __shfl_xor_sync(FULL, t, 2), gyp2 = __shfl_xor_sync(FULL, gy, 2),
                gzp2 = __shfl_xor_sync(FULL, gz, 2);
        const R t2  = w.g1 * t + w.g0 * tp + w.sgn_ih[1] * (gy + gyp2);
        const R gz2 = w.g1 * gz + w.g0 * gzp2;
        // stage z
        const R t2p = __shfl_xor_sync(FULL, t2, 4), gz2p = __shfl_xor_sync(FULL, gz2, 4);
        const R r   = w.g1 * t2 + w.g0 * t2p + w.sgn_ih[2] * (gz2 + gz2p);
        return r * w.JxW;
      }
    else
      {
        const R vp = __shfl_xor_sync(FULL, v, 1), gxp = __shfl_xor_sync(FULL, g[0], 1);
        const R gyp = __shfl_xor_sync(FULL, g[1], 1);
        const R t   = w.g1 * v + w.g0 * vp + w.sgn_ih[0] * (g[0] + gxp);
        const R gy  = w.g1 * g[1] + w.g0 * gyp;
        const R tp = __shfl_xor_sync(FULL, t, 2), gyp2 = __shfl_xor_sync(FULL, gy, 2);
        const R r  = w.g1 * t + w.g0 * tp + w.sgn_ih[1] * (gy + gyp2);
        return r * w.JxW;
      }
  }

  // Value-only integration butterfly: sum_q JxW v_q phi_l(x_q).
  template <int DIM, typename R>
  __device__ __forceinline__ R integrate_value_butterfly(R v, const QP<DIM, R> &w)
  {
    constexpr unsigned FULL = 0xffffffffu;
    R t = w.g1 * v + w.g0 * __shfl_xor_sync(FULL, v, 1);
    t   = w.g1 * t + w.g0 * __shfl_xor_sync(FULL, t, 2);
    if constexpr (DIM == 3)
      t = w.g1 * t + w.g0 * __shfl_xor_sync(FULL, t, 4);
    return t * w.JxW;
  }

  // (K u)_l for this lane's node l: the cell integral of grad phi_l . grad u_h,
  // exact on the uniform cell (the 2-point Gauss rule integrates it exactly).
  template <int DIM, typename R>
  __device__ __forceinline__ R stiffness_apply(const R *s, int b0, const QP<DIM, R> &w, const Grid &g)
  {
    R acc = kx<R>(g, 0) * s[b0 + w.koff[0]];
#pragma unroll
    for (int x = 1; x < (1 << DIM); ++x)
      acc += kx<R>(g, x) * s[b0 + w.koff[x]];
    return acc;
  }

  // Step 5 of the data flow: sum the per-cell node contributions
  // s_con[comp * CS + l * CP + cell] of the tile per box node (fixed order),
  // write nodes owned by the tile to dst and the others to the tile's slot of
  // the partial buffer (layout [tile][comp][BOX]).  With `mapped` (grain
  // cut-off), contribution row b belongs to component comp_of(b, gl) of the
  // c_all components; the owned nodes of the grains absent from the tile
  // (bit clear in tmask) are written as zero, their partial slots are left
  // alone (the combine step skips them).
  // With `epi` (the residual's epilogue hook) the owned nodes are stored as
  // (sum - sub) * scale; the partials stay raw (the combine step applies it).
  // LS = 2: s_con points at one lane of contributions held as packed pairs.
  template <int DIM, typename R, int LS = 1>
  __device__ __forceinline__ void sum_and_store(const R *s_con, int ncomp, const Grid &g, const TileCoord &tc,
                                                const BoxNode<DIM> &bn, R *__restrict__ dst, R *__restrict__ partial,
                                                unsigned long long gl = 0, bool mapped = false, int c_all = 0,
                                                unsigned tmask = 0, const ResidualHooks *epi = nullptr)
  {
    using T = Tile<DIM>;
    if (!bn.active || !bn.inside)
      return;
    // contributing (local node l, cell) pairs of this box node
    int  src_off[T::NQ];
    bool ok[T::NQ];
#pragma unroll
    for (int l = 0; l < T::NQ; ++l)
      {
        const int cx = bn.bx - (l & 1), cy = bn.by - ((l >> 1) & 1), cz = (DIM == 3) ? bn.bz - ((l >> 2) & 1) : 0;
        ok[l]      = cx >= 0 && cx < T::TX && cy >= 0 && cy < T::TY && cz >= 0 && cz < T::TZ;
        src_off[l] = (l * T::CP + (ok[l] ? cx + T::TX * (cy + T::TY * cz) : 0)) * LS;
      }
    const int gi = tc.o[0] + bn.bx, gj = tc.o[1] + bn.by, gk = (DIM == 3) ? tc.o[2] + bn.bz : 0;
    bool owned   = (bn.bx > 0 || gi == 0) && (bn.bx < T::TX || gi == g.n[0]) && (bn.by > 0 || gj == 0) &&
                 (bn.by < T::TY || gj == g.n[1]);
    if (DIM == 3)
      owned = owned && (bn.bz > 0 || gk == 0) && (bn.bz < T::TZ || gk == g.n[2]);
    R *out = owned ? dst + bn.gidx : partial + tc.linear * (mapped ? c_all : ncomp) * (long long)T::BOX + bn.b;
    const long long ost = owned ? g.ld : (long long)T::BOX;
    const bool      fin = owned && epi && epi->epilogue;
    // (v - sub) * scale for the owned entry of component cc
    auto finish = [&](R v, int cc) -> R {
      if (!fin)
        return v;
      const R sub = epi->subtract ? R(epi->subtract[cc * g.ld + bn.gidx]) : R(0);
      return (v - sub) * R(epi->scale);
    };
    for (int comp = bn.grp; comp < ncomp; comp += T::NG)
      {
        const R *sc  = s_con + comp * T::CS * LS;
        R        sum = R(0);
#pragma unroll
        for (int l = 0; l < T::NQ; ++l)
          if (ok[l])
            sum += sc[src_off[l]];
        const int cc = mapped ? comp_of(comp, gl) : comp;
        out[cc * ost] = finish(sum, cc);
      }
    if (mapped && owned)
      for (int comp = 2 + bn.grp; comp < c_all; comp += T::NG)
        if (((tmask >> (comp - 2)) & 1u) == 0u)
          out[comp * ost] = finish(R(0), comp);
  }

  // Interior-tile form of sum_and_store: the owned nodes are the ones on no
  // face of the box (np.inner), written at node0 + the fixed offset; the
  // others go to the tile's partial slot.
  template <int DIM, typename R, int LS = 1>
  __device__ __forceinline__ void sum_and_store_interior(const R *s_con, int ncomp, const Grid &g,
                                                         long long tile_linear, const NodePlan<DIM> &np,
                                                         long long node0, R *__restrict__ dst,
                                                         R *__restrict__ partial, unsigned long long gl = 0,
                                                         bool mapped = false, int c_all = 0, unsigned tmask = 0,
                                                         const ResidualHooks *epi = nullptr)
  {
    using T = Tile<DIM>;
    if (!np.active)
      return;
    const bool      owned = np.inner;
    R              *out   = owned ? dst + node0 + np.off
                                  : partial + tile_linear * (mapped ? c_all : ncomp) * (long long)T::BOX + np.b;
    const long long ost   = owned ? g.ld : (long long)T::BOX;
    const bool      fin   = owned && epi && epi->epilogue;
    auto finish = [&](R v, int cc) -> R {
      if (!fin)
        return v;
      const R sub = epi->subtract ? R(epi->subtract[cc * g.ld + node0 + np.off]) : R(0);
      return (v - sub) * R(epi->scale);
    };
    for (int comp = np.grp; comp < ncomp; comp += T::NG)
      {
        const R *sc  = s_con + (comp * T::CS + np.cbase) * LS;
        R        sum = R(0);
#pragma unroll
        for (int l = 0; l < T::NQ; ++l)
          if ((np.ok >> l) & 1u)
            sum += sc[(l * T::CP - ((l & 1) + T::TX * ((l >> 1) & 1) + T::TX * T::TY * ((l >> 2) & 1))) * LS];
        const int cc  = mapped ? comp_of(comp, gl) : comp;
        out[cc * ost] = finish(sum, cc);
      }
    if (mapped && owned)
      for (int comp = 2 + np.grp; comp < c_all; comp += T::NG)
        if (((tmask >> (comp - 2)) & 1u) == 0u)
          out[comp * ost] = finish(R(0), comp);
  }

  // Second pass of the scatter: nodes on an interior tile face sum the
  // partials of the 2, 4 or 8 tiles that share them, in a fixed order.  One
  // thread per (node, component): blockIdx.y is the component, so the
  // partial loads of different components are independent.
  // tile_mask (grain cut-off): a tile's partial of grain component 2 + b
  // exists only when bit b of tile_mask[tile] is set; nullptr = all exist.
  // epi (the residual's epilogue hook, nullptr for none): the combined sums
  // are stored as (sum - sub) * scale.
  // NC > 0: the component count at compile time, one thread per node, so a
  // thread's partial loads of all components can be in flight together (same
  // sums, same order).
  template <int DIM, typename R, int NC = 0>
  __global__ void __launch_bounds__(256) combine_kernel(const Grid g, int ncomp, const R *__restrict__ partial,
                                                        R *__restrict__ dst, const uint16_t *__restrict__ tile_mask,
                                                        const double *__restrict__ epi_sub = nullptr,
                                                        double epi_scale = 1.0, int epi = 0)
  {
    if constexpr (NC > 0)
      ncomp = NC;
    using T              = Tile<DIM>;
    const long long idx  = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int       comp = blockIdx.y;
    if (idx >= g.N)
      return;
    int c[3];
    if (g.N < (1ll << 31))
      {
        // multiply-shift instead of 64-bit division (most threads only classify their node)
        const unsigned q0 = fast_div(unsigned(idx), g.mnode[0], g.snode[0]);
        const unsigned q1 = fast_div(q0, g.mnode[1], g.snode[1]);
        c[0]              = int(unsigned(idx) - q0 * unsigned(g.nn[0]));
        c[1]              = int(q0 - q1 * unsigned(g.nn[1]));
        c[2]              = int(q1);
      }
    else
      {
        c[0] = int(idx % g.nn[0]);
        c[1] = int((idx / g.nn[0]) % g.nn[1]);
        c[2] = int(idx / ((long long)g.nn[0] * g.nn[1]));
      }
    const int TT[3]  = {T::TX, T::TY, T::TZ};
    int       nt[3]  = {1, 1, 1}; // number of candidate tiles per direction
    int       t0[3]  = {0, 0, 0}; // first candidate tile
    int       lo[3]  = {0, 0, 0}; // local box coordinate in the first candidate
    bool      shared = false;
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      {
        if (c[d] % TT[d] == 0 && c[d] > 0 && c[d] < g.n[d])
          {
            shared = true;
            nt[d]  = 2;
            t0[d]  = c[d] / TT[d] - 1;
            lo[d]  = TT[d];
          }
        else
          {
            t0[d] = min(c[d] / TT[d], g.nt[d] - 1);
            lo[d] = c[d] - t0[d] * TT[d];
          }
      }
    if (!shared)
      return;
    // the (up to 8) tiles sharing the node, in a fixed order: the node's slot
    // in each tile's partials and the grains each tile wrote
    long long slot[8];
    unsigned  tm[8];
    bool      has[8];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int bb = 0; bb < 2; ++bb)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc)
          {
            const int k = 4 * a + 2 * bb + cc;
            has[k]      = a < nt[2] && bb < nt[1] && cc < nt[0];
            const int       ti = t0[0] + cc, tj = t0[1] + bb, tk = t0[2] + a;
            const int       bx = lo[0] - cc * TT[0], by = lo[1] - bb * TT[1], bz = lo[2] - a * TT[2];
            const long long tile = ti + (long long)g.nt[0] * (tj + (long long)g.nt[1] * tk);
            slot[k] = tile * ncomp * (long long)T::BOX + bx + T::BX * (by + T::BY * bz);
            tm[k]   = (has[k] && tile_mask) ? unsigned(tile_mask[tile]) : ~0u;
          }
    // grains written by any of the sharing tiles: the others sum to zero
    // without a look at the candidates (most shared nodes of a packing lie
    // between tiles without a relevant grain)
    unsigned any = 0u;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (has[k])
        any |= tm[k];
    // NC > 0: one thread loops over all components (known at compile time);
    // otherwise in 2D one component per thread (blockIdx.y), in 3D the loop
    constexpr bool PER_COMP = DIM == 2 && NC == 0;
    const int      c_end    = PER_COMP ? comp + 1 : ncomp;
#pragma unroll
    for (int cp = PER_COMP ? comp : 0; cp < (NC > 0 ? NC : c_end); ++cp)
      {
        R sum = R(0);
        if (cp < 2 || ((any >> (cp - 2)) & 1u) != 0u)
          {
#pragma unroll
            for (int k = 0; k < 8; ++k)
              if (has[k] && (cp < 2 || ((tm[k] >> (cp - 2)) & 1u) != 0u))
                sum += partial[slot[k] + cp * (long long)T::BOX];
          }
        if (epi)
          sum = (sum - (epi_sub ? R(epi_sub[cp * g.ld + idx]) : R(0))) * R(epi_scale);
        dst[cp * g.ld + idx] = sum;
      }
  }
} // namespace sint
