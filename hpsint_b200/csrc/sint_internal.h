// Internal state of a sintering-operator context (not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/hpsint_b200.h"
#include "sint_common.cuh"

namespace sint
{
  void set_error(const std::string &msg);
  int  cuda_fail(cudaError_t e, const char *what);

  // Deterministic reductions: NB_RED fixed block partials, then one block.
  constexpr int NB_RED       = 592; // 4 x 148 SMs
  constexpr int MAX_MULTIDOT = 64;
  constexpr int RED_TICKETS  = 1; // doubles after the partials holding the last-block ticket counter
  // Elements per chunk of the grain cut-off's live-chunk map of Krylov vectors
  // (a multiple of the 128 elements one warp's 16-byte packs cover).
  constexpr long long LIVE_CHUNK = 1024;

  struct Workspace; // Newton/GMRES vectors, sint_newton.cu

  struct Ctx
  {
    sint_mesh   mesh;
    sint_params params;
    Grid        grid;
    Phys        phys;
    int         G = 0, C = 0;
    long long   N = 0, ld = 0;

    double *lin64 = nullptr; // linearisation point, C blocks
    float  *lin32 = nullptr; // FP32 shadow
    bool    has_lin = false;

    double *partial       = nullptr; // tile-face partial sums of the cell kernels
    size_t  partial_bytes = 0;

    // grain cut-off (SinteringOperatorData::set_component_mask,
    // operator_sintering_data.h:149-298): bit i of mask[cell] set when grain
    // i is relevant on the cell; the kernels use it while `cut` is set
    uint16_t *mask    = nullptr;
    long long n_cells = 0;
    bool      cut     = false;
    double    cut_tol = 0.0;
    bool      pc_cut  = false; // preconditioner diagonals with the cut-off too (else from the full operator)
    // tiles sorted into classes by their number of relevant grains (device)
    int                *cut_tiles  = nullptr; // tile ids, class by class
    unsigned long long *cut_grains = nullptr; // their packed grain lists
    uint16_t           *cut_union  = nullptr; // their union masks
    uint16_t           *tile_union = nullptr; // union mask by tile id (combine step)
    int                *cut_range  = nullptr; // class offsets, SINT_MAX_GRAINS + 2
    unsigned           *cut_count  = nullptr; // class sizes / scatter cursors, SINT_MAX_GRAINS + 1
    CutTiles            cut_view;             // the above as the kernels take them
    // nodes: the grains relevant on any adjacent cell; Krylov vectors: chunks
    // of LIVE_CHUNK elements that can be non-zero under the cut-off
    uint16_t *node_mask  = nullptr;
    uint32_t *live       = nullptr;
    bool      skip_zeros = true; // GMRES skips the chunks that are not live

    // grain-tracker particle detection (sint_tracker.cu): union-find parents
    // per cell, per-block root counts, accumulators per particle, error flag
    int                *seg_parent  = nullptr;
    int                *seg_blocks  = nullptr;
    unsigned long long *seg_acc     = nullptr;
    int                 seg_acc_cap = 0;
    int                *seg_error   = nullptr;

    // advection (sint_set_advection): the grains' segment of every cell and
    // the segments' velocities and centers, copied from the caller
    bool      adv          = false;
    int      *adv_cells    = nullptr; // G x n_cells
    double   *adv_segments = nullptr; // n_segments x 9 (velocity table)
    long long adv_seg_cap  = 0;       // capacities in elements
    unsigned *adv_error    = nullptr; // count of invalid ids
    AdvData   adv_view;               // the above as the kernels take them
    // the advection mechanism (sint_set_advection_mechanism): the table is
    // recomputed from the forces of every residual evaluation's state
    bool                  adv_mech      = false;
    sint_advection_params adv_prm       = {};
    double               *adv_centers   = nullptr; // n_segments x 3
    double               *adv_vft       = nullptr; // n_segments x (volume, force, torque)
    long long            *adv_off       = nullptr; // segment offsets (S + 1) and totals (S)
    unsigned             *adv_items     = nullptr; // (b, cell) items sorted by segment
    double               *adv_slots     = nullptr; // per-tile pieces of the force sums
    long long             adv_n_valid   = 0;       // items with a segment
    long long adv_cen_cap = 0, adv_vft_cap = 0, adv_off_cap = 0, adv_items_cap = 0, adv_slots_cap = 0;

    // preconditioner of the Cahn-Hilliard block: 0 = 2x2 node-block Jacobi,
    // 1 = symmetric Gauss-Seidel on the assembled block (sint_chsgs.cu)
    int     pc_kind   = 0;
    bool    has_ch    = false;   // the assembled block belongs to the current set-up
    double *ch_A64    = nullptr; // 3^dim x 4 blocks of ld: 2x2 blocks per node row and neighbour
    float  *ch_A32    = nullptr;
    double *ch_dinv64 = nullptr; // 4 blocks of ld: inverted centre blocks
    float  *ch_dinv32 = nullptr;

    double *pc_raw   = nullptr; // (G+4) blocks: CH 2x2 entries, AC diagonal
    double *pc_inv64 = nullptr; // (G+4) blocks: CH 2x2 inverse, AC inverse diagonal
    float  *pc_inv32 = nullptr;
    bool    has_pc   = false;

    double   *red        = nullptr; // reduction partials: (MAX_MULTIDOT + 1) x NB_RED doubles, then the ticket
    unsigned *red_ticket = nullptr; // blocks of a reduction that finished (the last one sums; back to 0)

    // DampedNewtonSolver state that outlives one solve (solvers_nonlinear.h:390-391)
    unsigned history_newton_iterations      = 0;
    unsigned history_linear_iterations_last = 0;

    Workspace *ws = nullptr;
  };

  // Reductions (sint_blas.cu); `out` is a device pointer.  `live` (grain
  // cut-off, GMRES vectors only): chunks whose bit is clear are zero in every
  // operand; read-only and update kernels skip them, kernels that produce a
  // vector write zeros there.  nullptr = everything live.
  int dot_f64(Ctx *c, long long n, const double *x, const double *y, double *out, cudaStream_t s);
  int dot_f32(Ctx *c, long long n, const float *x, const float *y, double *out, cudaStream_t s);
  // out[i] = <w, V + i * stride> for i < m (FP64 accumulation)
  template <typename R>
  int multidot(Ctx *c, long long n, const R *w, const R *V, long long stride, int m, double *out, cudaStream_t s,
               const uint32_t *live = nullptr);
  // w -= sum_i coef[i] * (V + i * stride), coef on the device
  template <typename R>
  int multiaxpy(long long n, R *w, const R *V, long long stride, int m, const double *coef, cudaStream_t s);
  // w -= sum_i coef[i] * V_i and norm2_out[0] = |w|^2 after the update (device scalar)
  template <typename R>
  int multiaxpy_norm2(Ctx *c, long long n, R *w, const R *V, long long stride, int m, const double *coef,
                      double *norm2_out, cudaStream_t s, const uint32_t *live = nullptr);
  // the same two, skipped on the device when *cond == 0 (launched unconditionally, decided on the GPU)
  template <typename R>
  int multidot_if(Ctx *c, long long n, const R *w, const R *V, long long stride, int m, double *out, const int *cond,
                  cudaStream_t s, const uint32_t *live = nullptr);
  template <typename R>
  int multiaxpy_norm2_if(Ctx *c, long long n, R *w, const R *V, long long stride, int m, const double *coef,
                         double *norm2_out, const int *cond, cudaStream_t s, const uint32_t *live = nullptr);
  // y = x / d_div[0] (divisor on the device)
  template <typename R>
  int scale_by_device(long long n, const R *x, const double *d_div, R *y, cudaStream_t s,
                      const uint32_t *live = nullptr);
  // y = a * x + b * y  (a, b on the host)
  template <typename R>
  int axpby(long long n, double a, const R *x, double b, R *y, cudaStream_t s, const uint32_t *live = nullptr);
  // y = sum_i y_i-combination: y = x + sum_i coef[i] * V_i (coef on the device), FP32/FP64 V
  template <typename R>
  int lincomb(long long n, R *y, const R *V, long long stride, int m, const double *coef, cudaStream_t s,
              const uint32_t *live = nullptr);
  template <typename S, typename D>
  int convert(long long n, const S *x, D *y, cudaStream_t s);

  int free_workspace(Ctx *c);

  // Validates and fills the operator description of c (no allocation).
  int describe_operator(const sint_mesh *mesh, const sint_params *params, Ctx *c);
  // Cell masks / tile classes the kernels use: with the cut-off on, else nullptr.
  inline const uint16_t *active_mask(const Ctx *c) { return c->cut ? c->mask : nullptr; }
  inline const uint16_t *preconditioner_mask(const Ctx *c) { return c->pc_cut ? active_mask(c) : nullptr; }
  inline const CutTiles *active_cut(const Ctx *c) { return c->cut ? &c->cut_view : nullptr; }
  inline const uint16_t *active_tile_union(const Ctx *c) { return c->cut ? c->tile_union : nullptr; }
  inline const uint32_t *active_live(const Ctx *c) { return (c->cut && c->skip_zeros) ? c->live : nullptr; }
  inline const AdvData  *active_adv(const Ctx *c) { return c->adv ? &c->adv_view : nullptr; }

  // The advection mechanism's update before a residual evaluation: forces of
  // u, then the velocity table (sint_advection.cu).
  int advection_update(Ctx *c, const double *u, cudaStream_t s);
  // The assembled Cahn-Hilliard block and its Gauss-Seidel sweeps
  // (sint_chsgs.cu): set-up at the linearisation point, and z_(c,mu) =
  // SGS(r_(c,mu)) on the first two blocks of z (the others untouched).
  int ch_sgs_setup(Ctx *c, cudaStream_t s);
  template <typename R>
  cudaError_t ch_sgs_apply(const Ctx *c, const R *r, R *z, cudaStream_t s);
  // J v through the cell kernel + combine, with c->partial as scratch.
  template <typename R>
  cudaError_t dispatch_jvp(const Ctx *c, const R *lin, const R *src, R *dst, cudaStream_t s);
} // namespace sint

struct sint_ctx : public sint::Ctx
{};
