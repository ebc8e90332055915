/*
 * hpsint_b200: B200-native matrix-free sintering operator (C ABI).
 *
 * The operator is hpsint's coupled Cahn-Hilliard / Allen-Cahn system in
 * (c, mu, eta_1 .. eta_G) on uniform Cartesian Q1 meshes (2D quads, 3D hexes),
 * QGauss(2) quadrature, Wang bulk free energy, scalar or tensorial
 * volume/vapour/surface/grain-boundary mobility.
 *
 * Conventions shared by every entry point
 *   - All vector pointers are DEVICE pointers owned by the caller.
 *   - A block vector ("DoF vector") holds C = G + 2 blocks; block b starts at
 *     element b * block_stride and holds the N nodal values of component b
 *     (c, mu, eta_1, .., eta_G) in lexicographic node order: x fastest, then y,
 *     then z.  sint_dof_layout() reports N, C and block_stride; entries
 *     between N and block_stride are never read and are written as zero by the
 *     BLAS-1 routines only.  Device pointers must be 16-byte aligned.
 *   - Every call is asynchronous on `stream` (a cudaStream_t; NULL = legacy
 *     default stream) unless it says otherwise.
 *   - Every call returns a sint_status; no C++ exception crosses the ABI.
 *   - A context is not re-entrant: calls on one context must not overlap
 *     (the reference operator is single-threaded per MPI rank as well).
 */
#ifndef HPSINT_B200_H
#define HPSINT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SINT_MAX_GRAINS 12
#define SINT_ABI_VERSION 1

typedef struct CUstream_st *sint_stream_t; /* identical to cudaStream_t */
typedef struct sint_ctx     sint_ctx;

typedef enum
{
  SINT_OK                 = 0,
  SINT_ERR_ARG            = 1, /* null pointer, bad size or misaligned pointer */
  SINT_ERR_GRAINS         = 2, /* n_grains outside [1, SINT_MAX_GRAINS];
                                  instantiation.h:61-68 ExcInvalidNumberOfComponents */
  SINT_ERR_CUDA           = 3, /* a CUDA runtime call failed; see sint_last_error() */
  SINT_ERR_NOT_READY      = 4, /* e.g. vmult before a linearisation point was set */
  SINT_ERR_NO_CONVERGENCE = 5, /* linear solver did not converge:
                                  deal.II SolverControl::NoConvergence */
  SINT_ERR_NEWTON         = 6, /* damped Newton failed: solvers_nonlinear.h:183-206
                                  ExcNewtonDidNotConverge ("Newton" or "damping") */
  SINT_ERR_NONFINITE      = 7, /* NaN/Inf in a residual norm */
  SINT_ERR_DT_MIN         = 8  /* time step fell below the minimum (driver.h:2189-2191) */
} sint_status;

/* Uniform Cartesian mesh: n_cells[d] cells of size h[d] in direction d
 * (entries d >= dim are ignored).  Replaces the reference's
 * create_mesh_from_divisions / subdivided_hyper_rectangle
 * (include/pf-applications/grid/grid_tools.h:698-719) with no constraints. */
typedef struct
{
  int    dim;
  int    n_cells[3];
  double h[3];
  double origin[3];
} sint_mesh;

/* Model parameters.  A, B: FreeEnergy(A, B) (sintering/free_energy.h:187-190);
 * kappa_c, kappa_p: SinteringOperatorData (operator_sintering_data.h:51-62);
 * Mvol..L: ProviderAbstract (mobility.h:45-76); tensorial selects
 * MobilityTensorial instead of MobilityScalar (operator_sintering_data.h:38-49). */
typedef struct
{
  int    n_grains;
  double A, B;
  double kappa_c, kappa_p;
  double Mvol, Mvap, Msurf, Mgb, L;
  int    tensorial;
} sint_params;

/* ---------------------------------------------------------------------- */
/* Operator: SinteringOperatorGeneric                                      */
/* (applications/sintering/include/pf-applications/sintering/              */
/*  operator_sintering_generic.h:323-1085)                                 */

/* SinteringOperatorGeneric::create (operator_sintering_generic.h:369-391),
 * with the MatrixFree set-up for the uniform mesh. */
int sint_create(const sint_mesh *mesh, const sint_params *params, sint_ctx **ctx);

/* Releases every device buffer owned by the context (synchronises first). */
int sint_destroy(sint_ctx *ctx);

/* OperatorBase::initialize_dof_vector (sintering/operator_base.h:143-149):
 * reports the block-vector layout the operator expects. */
int sint_dof_layout(const sint_ctx *ctx, int64_t *n_nodes, int *n_components, int64_t *block_stride);

/* TimeIntegratorData weights (time_integration/time_integrator_data.h:150-163):
 * w0 = primary weight, w_hist[0..order-1] = weights[1..order] applied to the old
 * solutions, w_alg = algebraic weight of the mu row (1 for implicit schemes).
 * order <= 3 (BDF1..BDF3, time_schemes.h:64-153). */
int sint_set_time_weights(sint_ctx *ctx, double w0, const double *w_hist, int order, double w_alg);

/* Mobility::update (sintering/mobility.h:224-234): new mobility coefficients,
 * e.g. from ProviderRealistic at the new time. */
int sint_set_mobility(sint_ctx *ctx, double Mvol, double Mvap, double Msurf, double Mgb, double L);

/* SinteringOperatorData::fill_quadrature_point_values
 * (sintering/operator_sintering_data.h:300-409).  Instead of caching values
 * and gradients at quadrature points, the context copies the nodal state u
 * (C blocks) and an FP32 shadow of it; both are re-evaluated on the fly. */
int sint_set_linearization_point(sint_ctx *ctx, const double *u, sint_stream_t stream);

/* SinteringOperatorGeneric::evaluate_nonlinear_residual<with_time_derivative>
 * (operator_sintering_generic.h:393-448): dst = R(src).  with_time_derivative:
 * 0 drops the time terms, 1 keeps w0*u only, 2 adds the BDF history
 * sum_i w_hist[i] * hist[i].  hist is a HOST array of `order` device pointers
 * to old solutions (SolutionHistory::get_old_solutions); ignored unless
 * with_time_derivative == 2.  dst is overwritten. */
int sint_residual_f64(sint_ctx *ctx, double *dst, const double *src, const double *const *hist,
                      int with_time_derivative, sint_stream_t stream);

/* The residual's range hooks in device form.  evaluate_nonlinear_residual
 * (operator_sintering_generic.h:393-401) takes pre_operation and
 * post_operation callbacks that the cell loop calls on ranges of dst before
 * and after writing them; the reference's Jacobian-free operator uses them to
 * perturb the state and form a finite-difference quotient in the same pass
 * (lac/jacobian_operator.h:160-232).  Host callbacks cannot run inside the
 * device cell loop, so this entry point offers that use as data:
 *   dst = scale * (R(src + perturb_scale * perturb) - subtract)
 * with the perturbation formed while the node boxes are staged (src is not
 * modified and no perturbed vector is stored) and the epilogue fused into
 * the stores and the combine step (on periodic meshes it follows the
 * condensation of the slave rows as one extra pass).  perturb and subtract
 * may be NULL (no perturbation; subtract zero); perturb_scale = 0 and scale
 * = 1 leave the plain residual.  The pre_operation's zeroing of dst is
 * implied: every entry of dst is written.  Not with the advection mechanism
 * and a perturbation (SINT_ERR_ARG: the forces would need the perturbed
 * state).  dst must not alias perturb or subtract. */
typedef struct
{
  const double *perturb;
  double        perturb_scale;
  const double *subtract;
  double        scale;
} sint_residual_hooks;

int sint_residual_f64_hooks(sint_ctx *ctx, double *dst, const double *src, const double *const *hist,
                            int with_time_derivative, const sint_residual_hooks *hooks, sint_stream_t stream);

/* OperatorBase::vmult -> SinteringOperatorGeneric::vmult_internal
 * (operator_base.h:294-353, operator_sintering_generic.h:539-606):
 * dst = J(u_lin) src in FP64.  dst is overwritten. */
int sint_jvp_f64(sint_ctx *ctx, double *dst, const double *src, sint_stream_t stream);

/* Same product in FP32 with FP32 accumulation, linearised at the FP32 shadow. */
int sint_jvp_f32(sint_ctx *ctx, float *dst, const float *src, sint_stream_t stream);

/* Allocation-free FP64 Jacobian-vector product (no counterpart in the
 * reference).  For callers that may not call cudaMalloc -- e.g. code running
 * under another framework's memory pool, inside stream callbacks, or embedded
 * solvers with a fixed memory budget: no context is needed and nothing is
 * allocated.  The caller passes the mesh, the parameters, the time weights
 * (w0, w_alg as in sint_set_time_weights), the linearisation point `lin` and
 * the direction `src` (C blocks each, the layout sint_dof_layout reports) and
 * owns `dst`; the result equals sint_jvp_f64 on a context with the same state.
 * The product's only scratch, the partial sums on tile faces, lives in a
 * fixed device array of SINT_NOALLOC_SCRATCH_BYTES that every GPU loading the
 * library holds until exit; meshes needing more return SINT_ERR_ARG.  The
 * need is 600 * (G + 2) bytes per 4 x 4 x 2 cells in 3D and 648 * (G + 2)
 * bytes per 8 x 8 cells in 2D: with G = 4, up to 64 x 64 x 36 cells in 3D or
 * 520 x 520 cells in 2D.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current, so make it before any
 * stream capture.  That address is kept per device ordinal for the life of
 * the process: after a device reset (cudaDeviceReset) the process must not
 * call this entry point on that device again.  All calls share the array:
 * calls that overlap on the GPU (different streams, or different host
 * threads) race and give wrong results. */
#define SINT_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int sint_jvp_f64_noalloc(const sint_mesh *mesh, const sint_params *params, double w0, double w_alg,
                         const double *lin, const double *src, double *dst, sint_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Preconditioner: BlockPreconditioner2 (sintering/preconditioners.h:978-1343) */

/* BlockPreconditioner2::do_update (preconditioners.h:1260-1283) at the current
 * linearisation point.  Block 0 (c, mu): the inverse of each node's 2x2
 * diagonal block of the OperatorCahnHilliard tangent (preconditioners.h:85-169),
 * a point-block Jacobi in the spirit of InverseComponentBlockDiagonalMatrix
 * (lac/preconditioners.h:217-315) in place of the reference's ILU.
 * Block 1 (eta): InverseDiagonalMatrix of OperatorAllenCahn
 * (preconditioners.h:342-414, lac/preconditioners.h:159-213,
 * operator_base.h:364-389).  Kept in FP64 and FP32.  With advection set, both
 * blocks include the advection terms of the current velocity table
 * (precondition_advection_ch / _ac, operator_sintering_generic.h:800-850); on a
 * periodic mesh the slave rows are condensed into their masters and get the
 * identity. */
int sint_precond_setup(sint_ctx *ctx, sint_stream_t stream);

/* Block 0 of the preconditioner (BlockPreconditioner2Data::block_0,
 * preconditioner_parameters.h; default "ILU" in the reference):
 *   0  the 2x2 node-block Jacobi above (this library's default);
 *   1  the assembled Cahn-Hilliard block (OperatorCahnHilliard through
 *      MyMatrixFreeTools::compute_matrix, matrix_free/tools.h:29-175: 2x2
 *      blocks of every node row for its 3^dim neighbours) applied by one
 *      symmetric Gauss-Seidel sweep pair in multicolour order (nodes coloured
 *      by index parity), the GPU-parallel stand-in for the reference's ILU(0)
 *      (lac/preconditioners.h:607-1088).  The grain block keeps the inverse
 *      diagonal.  Not available with periodic constraints (set-up returns
 *      SINT_ERR_ARG).  Pairs best with right-preconditioned GMRES
 *      (sint_newton_params.right_preconditioning): with left preconditioning
 *      GMRES stops on a residual dominated by the Cahn-Hilliard rows.
 * Takes effect at the next sint_precond_setup; type 1 allocates the matrix
 * (3^dim x 4 FP64 + FP32 values per node) at its first set-up. */
int sint_set_preconditioner_type(sint_ctx *ctx, int type);

/* The assembled Cahn-Hilliard block of preconditioner type 1: 3^dim x 4
 * blocks of block_stride (device), A[(k * 4 + e) * block_stride + n] = entry e
 * (J_cc, J_c,mu, J_mu,c, J_mu,mu) of node n's row for its neighbour k =
 * (dx + 1) + 3 (dy + 1) (+ 9 (dz + 1)).  Requires sint_precond_setup first. */
int sint_ch_matrix_f64(sint_ctx *ctx, double *A, sint_stream_t stream);

/* BlockPreconditioner2::vmult (preconditioners.h:1222-1258): z = P^-1 r. */
int sint_precond_apply_f64(sint_ctx *ctx, double *z, const double *r, sint_stream_t stream);
int sint_precond_apply_f32(sint_ctx *ctx, float *z, const float *r, sint_stream_t stream);

/* OperatorBase::compute_inverse_diagonal of OperatorAllenCahn
 * (operator_base.h:364-389): G blocks of block_stride, 1/d where |d| > 1e-10,
 * else 1.  Requires sint_precond_setup first. */
int sint_ac_inverse_diagonal_f64(sint_ctx *ctx, double *inv_diag, sint_stream_t stream);

/* The assembled (not inverted) 2x2 node blocks of the Cahn-Hilliard tangent,
 * 4 blocks of block_stride: J_cc, J_c,mu, J_mu,c, J_mu,mu (row = tested
 * equation, column = unknown).  Requires sint_precond_setup first. */
int sint_ch_blocks_f64(sint_ctx *ctx, double *blocks, sint_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Grain cut-off: SinteringOperatorData::set_component_mask                 */
/* (operator_sintering_data.h:149-298), called by the driver before every   */
/* step attempt with the current solution when GrainCutOffTolerance != 0    */
/* (driver.h:2212-2218, parameters.h:314, :421).                            */
/* ---------------------------------------------------------------------- */

/* Marks grain b relevant on a cell when max |eta_b| over the cell's nodes
 * exceeds tol (u: C blocks of block_stride, device).  While set, the
 * context's residual, both Jacobian-vector products and the Newton solver
 * restrict every cell to its relevant grains (the context-free
 * sint_jvp_f64_noalloc always applies the full operator), as
 * do_evaluate_nonlinear_residual_nt and
 * do_vmult_range_no_template (operator_sintering_generic.h:456-537,
 * :1008-1081) and the Allen-Cahn preconditioner block
 * (preconditioners.h:787-817, :865-882) do: an absent grain contributes
 * nothing to the cell's sums and its row receives nothing from the cell.
 * The preconditioner's diagonals come from the full operator unless
 * sint_set_preconditioner_cut_off switches the cut-off on for them too.
 * The reference forms the union over the cells of one SIMD batch; this
 * library keeps one set per cell.  tol == 0 switches the cut-off off;
 * tol < 0 is SINT_ERR_ARG.  The first call allocates one uint16 per cell. */
int sint_set_component_mask(sint_ctx *ctx, const double *u, double tol, sint_stream_t stream);

/* Whether sint_precond_setup applies the grain cut-off as well (on != 0):
 * the Allen-Cahn diagonal then drops absent grains' contributions and empty
 * diagonals invert to 1, as the reference's matrix-based block does
 * (preconditioners.h:787-817, :865-882).  Default off: the block-Jacobi
 * diagonals come from the full operator, which changes only how fast GMRES
 * converges (at a grain's cut boundary the assembled-from-relevant-cells
 * rows are poorly scaled by their partial diagonals), not the Newton system
 * or its solution.  Takes effect at the next sint_precond_setup. */
int sint_set_preconditioner_cut_off(sint_ctx *ctx, int on);

/* Copies u_old into u (both C blocks, device) on the DoFs the cut-off takes
 * out of the system: grain b at a node none of whose cells has b relevant.
 * Those DoFs get no residual, Jacobian or preconditioner entry, so Newton
 * keeps whatever the initial guess holds there; a caller that starts Newton
 * from a predicted guess (the reference's predictor hook, driver.h:2001-2058)
 * calls this so they keep their old values instead of the extrapolation (no
 * counterpart in the reference).  SINT_ERR_NOT_READY without a cut-off. */
int sint_cut_off_freeze(sint_ctx *ctx, double *u, const double *u_old, sint_stream_t stream);

/* Whether the device GMRES (sint_newton_solve) skips, under the cut-off, the
 * chunks of its vectors that are zero by construction: a grain's DoF at a
 * node none of whose cells has the grain relevant receives no residual,
 * Jacobian or preconditioner entry.  Results are bitwise the same either
 * way; default on (no counterpart in the reference, whose vectors are dense
 * as well). */
int sint_set_cut_off_skip_zero_chunks(sint_ctx *ctx, int on);

/* The "Cut-off statistic" (operator_sintering_data.h:236-296): counts[k]
 * (host, n_grains + 1 entries) = number of cells with k relevant grains.
 * SINT_ERR_NOT_READY without a cut-off.  Synchronises `stream`. */
int sint_component_mask_statistics(sint_ctx *ctx, int64_t *counts, sint_stream_t stream);

/* Copies the cell masks (bit b = grain b relevant; n_cells[0] * n_cells[1]
 * * n_cells[2] entries, x fastest) to the device array dst. */
int sint_get_component_mask(const sint_ctx *ctx, uint16_t *dst, sint_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Grain tracker: particle detection of one order parameter                 */
/* (GrainTracker::Tracker, grain_tracker/tracker.h:1195-1300).              */
/* ---------------------------------------------------------------------- */

/* run_flooding / detect_local_particle_groups
 * (grain_tracker/distributed_stitching.h:41-100, :441-480): a cell belongs
 * to a particle when the largest of its nodal values of `eta` (one block, N
 * values, device) exceeds threshold_lower (GrainTrackerData::threshold_lower,
 * default 0.01, sintering/parameters.h:98); particles are face-connected
 * sets of such cells.  particle_ids (device, n_cells[0] * n_cells[1] *
 * n_cells[2] ints, x fastest) receives each cell's particle number or -1;
 * particles are numbered in the order a lexicographic cell loop reaches them
 * (the reference numbers them in deal.II's cell order, and renumbers across
 * processes).  *n_particles (host) = their number.  Synchronises `stream`. */
int sint_grain_segments(sint_ctx *ctx, const double *eta, double threshold_lower, int *particle_ids,
                        int *n_particles, sint_stream_t stream);

/* The spherical representation's particle properties, per particle (host,
 * n_particles rows of 3 + dim doubles): measure, center[dim] (measure-
 * weighted cell centers, compute_particles_info, distributed_stitching.h:
 * 264-320), radius (largest |cell barycenter - center| + cell diameter / 2,
 * compute_particles_radii, :322-360) and the largest nodal value (the
 * particle max_value of run_flooding, :77-86).  Synchronises `stream`. */
int sint_grain_segment_properties(sint_ctx *ctx, const double *eta, const int *particle_ids, int n_particles,
                                  double *props, sint_stream_t stream);

/* Periodicity between particles (tracker.h:1290-1353): the distinct pairs
 * (p, q), p <= q, of particles of `particle_ids` (DEVICE, as returned by
 * sint_grain_segments) that own cells facing each other across a periodic
 * boundary of the context (sint_set_periodicity), in increasing order, into
 * the HOST array pairs[2 * max_pairs].  The tracker groups connected
 * particles into one grain of several segments (PeriodicityGraph::
 * build_groups).  More pairs than max_pairs: SINT_ERR_ARG with the count in
 * *n_pairs.  Synchronises `stream`. */
int sint_grain_segment_periodicity(sint_ctx *ctx, const int *particle_ids, int *pairs, int max_pairs, int *n_pairs,
                                   sint_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Periodic constraints (DoFTools::make_periodicity_constraints, driver.h:  */
/* 629-643; OperatorBase::vmult's constrained rows, operator_base.h:        */
/* 294-353).                                                                */

/* Makes the mesh periodic in the directions whose bit is set (bit d =
 * direction d; each needs >= 2 cells).  The nodes at coordinate n_cells[d]
 * become slaves of the nodes at 0: the residual, J v and the preconditioner
 * read the masters' values there, add the slave rows to the master rows,
 * and give the slave rows zero (residual) or the identity (J v,
 * preconditioner).  sint_newton_solve distributes the solution at the end.
 * 0 switches periodicity off.  The grain cut-off's masks and the advection
 * forces read the masters too; the grain tracker reads the nodal values as
 * they are (pass distributed vectors, as hpsint's tracker gets). */
int sint_set_periodicity(sint_ctx *ctx, unsigned directions);

/* AffineConstraints::distribute: every slave entry of u (all components)
 * takes its master's value. */
int sint_distribute_constraints(sint_ctx *ctx, double *u, sint_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Advection: rigid-body motion of the grains (AdvectionMechanism,          */
/* sintering/advection.h:297-520).  Replaces the AdvectionMechanism the     */
/* operator is constructed with (operator_sintering_generic.h:347-361).     */

/* Sets the grains' velocities for the residual and J v of this context
 * (operator_sintering_generic.h:167-177, :1015-1036: the c row gains
 * -(v_i c, grad phi) and the eta_i row -(v_i eta_i, grad phi) for every
 * grain i with a velocity on the cell).
 *   cell_segments  DEVICE, n_grains x n_cells int32 (cells x fastest): the
 *                  segment (particle) of order parameter b that cell belongs
 *                  to, -1 for none (AdvectionMechanism::cell_index_values,
 *                  advection.h:411-446)
 *   segments       DEVICE, n_segments x 9 doubles: translational velocity
 *                  (3), angular velocity (3; only z is used in 2D) and
 *                  center (3) of each segment; the velocity at x is
 *                  v_t + w x (x - center) (calc_translation_velocity /
 *                  calc_rotation_velocity, advection.h:330-352)
 * Both are copied (the caller may free or reuse its buffers); ids outside
 * [-1, n_segments) are an error.  cell_segments == NULL switches advection
 * off.  Synchronises `stream` (the id check). */
int sint_set_advection(sint_ctx *ctx, const int32_t *cell_segments, const double *segments, int n_segments,
                       sint_stream_t stream);

/* Parameters of the advection mechanism (AdvectionData,
 * sintering/parameters.h:719-745): Wang stiffness k, grain-boundary
 * threshold cgb, equilibrium concentration ceq, smoothening of the
 * grain-boundary filter, translation and rotation factors mt and mr. */
typedef struct
{
  double k, cgb, ceq, smoothening, mt, mr;
} sint_advection_params;

/* The advection mechanism with state-dependent velocities: every residual
 * evaluation of the context (sint_residual_f64 and the device Newton's)
 * first evaluates the segments' volumes, forces and torques from its input
 * state (AdvectionOperatorGeneric::evaluate_forces, operator_advection.h:
 * 86-373) and turns them into the velocity table (v_t = mt F / V,
 * w = mr T / V); J v uses the table of the latest evaluation, as
 * ResidualWrapperAdvection does (residual_wrapper.h:36-84).
 *   cell_segments  DEVICE, n_grains x n_cells int32 as for sint_set_advection
 *   centers        DEVICE, n_segments x 3: the segment centers (the grain
 *                  tracker's), about which torques and rotations are taken
 * Sums are deterministic (a fixed order independent of thread scheduling).
 * Synchronises `stream`.  cell_segments == NULL switches advection off;
 * sint_set_advection replaces the mechanism by fixed velocities. */
int sint_set_advection_mechanism(sint_ctx *ctx, const int32_t *cell_segments, const double *centers, int n_segments,
                                 const sint_advection_params *params, sint_stream_t stream);

/* Evaluates the forces of the state u and updates the velocity table; with
 * vft != NULL also copies the per-segment volume, force and torque to it
 * (DEVICE, n_segments rows of 1 + dim + (dim == 3 ? 3 : 1) doubles; 2D
 * torque = hpsint's scalar cross product r[1] F[0] - r[0] F[1]). */
int sint_advection_forces(sint_ctx *ctx, const double *u, double *vft, sint_stream_t stream);

/* CFLChecker::check_courant (sintering/cfl_checker.h:62-128) with the
 * current velocity table: *ok = 1 when |v| dt < cell diameter at every
 * quadrature point of every cell for every (relevant) grain with a
 * velocity there, else 0 (the driver then throws
 * ExcCourantConditionViolated).  Synchronises `stream`. */
int sint_advection_check_courant(sint_ctx *ctx, double dt, int *ok, sint_stream_t stream);

/* ---------------------------------------------------------------------- */
/* BLAS-1 on block vectors: DynamicBlockVector                              */
/* (include/pf-applications/lac/dynamic_block_vector.h:346-516).            */
/* n = number of elements (C * block_stride for a whole block vector).      */
/* Reductions accumulate in FP64 and write one double to a DEVICE pointer;  */
/* they use the context's reduction workspace (fixed block partials summed  */
/* in a fixed order, so results are bitwise reproducible).                  */

int sint_vec_axpy_f64(int64_t n, double a, const double *x, double *y, sint_stream_t stream); /* y += a x  (add) */
int sint_vec_sadd_f64(int64_t n, double s, double a, const double *x, double *y,
                      sint_stream_t stream);                                           /* y = s y + a x (sadd) */
int sint_vec_scale_f64(int64_t n, double a, double *x, sint_stream_t stream);          /* x *= a */
int sint_vec_dot_f64(sint_ctx *ctx, int64_t n, const double *x, const double *y, double *result,
                     sint_stream_t stream);                                                    /* operator* */
int sint_vec_norm2_f64(sint_ctx *ctx, int64_t n, const double *x, double *result, sint_stream_t stream); /* l2_norm */
int sint_vec_axpy_f32(int64_t n, float a, const float *x, float *y, sint_stream_t stream);
int sint_vec_dot_f32(sint_ctx *ctx, int64_t n, const float *x, const float *y, double *result, sint_stream_t stream);
int sint_vec_norm2_f32(sint_ctx *ctx, int64_t n, const float *x, double *result, sint_stream_t stream);
int sint_vec_f64_to_f32(int64_t n, const double *x, float *y, sint_stream_t stream);   /* FP32 shadow */
int sint_vec_f32_to_f64(int64_t n, const float *x, double *y, sint_stream_t stream);
/* out = (*norm_a <= *norm_b) ? a : b, decided on the device (norms are device
 * scalars, e.g. from sint_vec_norm2_f64); out may alias a or b. */
int sint_vec_select_f64(int64_t n, const double *a, const double *b, const double *norm_a, const double *norm_b,
                        double *out, sint_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Nonlinear solve: DampedNewtonSolver (lac/solvers_nonlinear.h:236-394)     */
/* with GMRES (lac/solvers_linear.h:57-117, deal.II SolverGMRES, classical  */
/* Gram-Schmidt) and BlockPreconditioner2, all on the device.              */

typedef struct
{
  /* NonLinearData (lac/solvers_nonlinear_parameters.h:40-60) */
  int    nl_max_iter;          /* 10 */
  double nl_abs_tol;           /* 1e-20 */
  double nl_rel_tol;           /* 1e-5 */
  int    l_max_iter;           /* 1000 */
  double l_abs_tol;            /* 1e-10 */
  double l_rel_tol;            /* 1e-2 */
  int    gmres_restart;        /* 30 (deal.II max_n_tmp_vectors) */
  int    threshold_newton_iter;/* 100: rebuild preconditioner every this many Newton its */
  int    threshold_linear_iter;/* 20: ... or when the last solve took more linear its */
  int    use_damping;          /* 1 */
  int    reuse_preconditioner; /* 1 */
  int    inner_precision;      /* 64: FP64 GMRES/Jacobian/preconditioner,
                                  32: FP32 Arnoldi vectors, Jacobian and
                                  preconditioner with FP64 dots and norms */
  int    right_preconditioning;/* 0: left preconditioning (deal.II SolverGMRES's
                                  default, as the reference); 1: right
                                  preconditioning, J P^-1 y = b, x = P^-1 y:
                                  GMRES stops on the true residual */
} sint_newton_params;

typedef struct
{
  int    newton_iterations;
  int    linear_iterations;
  int    residual_evaluations;
  int    jacobian_setups;
  int    preconditioner_setups;
  double initial_residual;
  double final_residual;
} sint_newton_stats;

/* Fills the reference defaults listed above. */
void sint_newton_default_params(sint_newton_params *p);

/* DampedNewtonSolver::clear (solvers_nonlinear.h:359-364): forgets the Newton
 * and linear iteration history that decides when the preconditioner is rebuilt
 * (the driver calls it after a failed step, driver.h:2193-2195). */
int sint_newton_clear(sint_ctx *ctx);

/* DampedNewtonSolver::solve (solvers_nonlinear.h:247-357) for R(u) = 0 with the
 * time weights already set: u (device, C blocks) is the initial guess on entry
 * and the solution on SINT_OK.  hist: HOST array of `order` device pointers
 * (residual history term, with_time_derivative = 2).  On SINT_ERR_NEWTON or
 * SINT_ERR_NO_CONVERGENCE u holds the last iterate.  Synchronises `stream`. */
int sint_newton_solve(sint_ctx *ctx, double *u, const double *const *hist, const sint_newton_params *params,
                      sint_newton_stats *stats, sint_stream_t stream);

/* ---------------------------------------------------------------------- */

/* ---------------------------------------------------------------------- */
/* Learned Newton initial guess (no counterpart in the reference: it plugs  */
/* in at the driver's predictor hook, sintering/driver.h:2001-2058).  FP32 */
/* building blocks of a grain-permutation-equivariant convolutional net;    */
/* tensors are NCHW float32 device arrays, grain streams of sample b are    */
/* batch entries b * G + i.  All calls are asynchronous on `stream`.        */

/* out[b][co] (+)= bias[co] + sum_ci w[co][ci] (*) in[b][ci]: 3x3, zero padding,
 * stride 1.  bias may be NULL; accumulate != 0 adds to out. */
int sint_nn_conv3x3_f32(const float *in, int B, int Cin, int H, int W, const float *w, const float *bias,
                        float *out, int Cout, int accumulate, sint_stream_t stream);
/* The same convolution on the tensor cores (tcgen05.mma kind::tf32, FP32
 * accumulation in TMEM) for 1 <= Cin <= 32 and 1 <= Cout <= 32: products of TF32
 * operands (FP32 values with the low 13 mantissa bits ignored).  status: a
 * device int the caller zeroes; set to 1 if a wait for the tensor core timed
 * out (the output is then incomplete). */
int sint_nn_conv3x3_tc_f32(const float *in, int B, int Cin, int H, int W, const float *w, const float *bias,
                           float *out, int Cout, int accumulate, int *status, sint_stream_t stream);
/* The same with a fused epilogue for inference: out = act(conv + bias
 * (+ out if accumulate) (+ addend[b / addend_group] if addend)), act = leaky
 * ReLU with `slope` if leaky != 0.  addend: [B / addend_group][Cout][H][W]
 * (the shared-stream term broadcast to the grain streams). */
int sint_nn_conv3x3_tc_ex_f32(const float *in, int B, int Cin, int H, int W, const float *w, const float *bias,
                              float *out, int Cout, int accumulate, const float *addend, int addend_group,
                              int leaky, float slope, int *status, sint_stream_t stream);
/* wT[ci][co][8 - k] = w[co][ci][k]: the kernel whose convolution with the
 * output gradient is the input gradient. */
int sint_nn_conv3x3_flip_f32(const float *w, int Cout, int Cin, float *wT, sint_stream_t stream);
/* floats of workspace sint_nn_conv3x3_wgrad_f32 needs for these sizes */
int64_t sint_nn_conv3x3_wgrad_workspace(int B, int Cin, int Cout, int H, int W);
/* dw[co][ci][k] (+)= sum_{b,pixels} dout[b][co] in[b][ci] shifted by tap k;
 * db[co] (+)= sum dout[b][co] (db may be NULL).  Deterministic. */
int sint_nn_conv3x3_wgrad_f32(const float *in, const float *dout, int B, int Cin, int Cout, int H, int W, float *dw,
                              float *db, int accumulate, float *work, sint_stream_t stream);
int sint_nn_leaky_relu_f32(int64_t n, float slope, const float *x, float *y, sint_stream_t stream);
/* dx = dy * f'(pre); dx may alias dy */
int sint_nn_leaky_relu_bwd_f32(int64_t n, float slope, const float *pre, const float *dy, float *dx,
                               sint_stream_t stream);
/* P[b] = sum_i h[b G + i] over tensors of chw elements per entry */
int sint_nn_grain_sum_f32(const float *h, int B, int G, int64_t chw, float *P, sint_stream_t stream);
/* Z[b G + i] += Q[b] */
int sint_nn_grain_bcast_add_f32(const float *Q, int B, int G, int64_t chw, float *Z, sint_stream_t stream);
/* Adam (Kingma & Ba 2015) with bias correction at step >= 1 */
int sint_nn_adam_f32(int64_t n, float *param, const float *grad, float *m, float *v, float lr, float beta1,
                     float beta2, float eps, int step, sint_stream_t stream);
/* out = w (pred - target) elementwise (weight may be NULL = 1) */
int sint_nn_weighted_diff_f32(int64_t n, const float *pred, const float *target, const float *weight, float *out,
                              sint_stream_t stream);
/* y += alpha a x elementwise (a may be NULL = 1) */
int sint_nn_mul_add_f32(int64_t n, float alpha, const float *a, const float *x, float *y, sint_stream_t stream);
/* doubles of workspace sint_nn_mse_f32 needs */
int64_t sint_nn_mse_workspace(void);
/* loss[0] = sum w (pred - target)^2 / n (weight may be NULL = 1); grad (may be
 * NULL) = 2 w (pred - target) / n.  Deterministic. */
int sint_nn_mse_f32(int64_t n, const float *pred, const float *target, const float *weight, float *grad,
                    double *loss, double *work, sint_stream_t stream);
/* Network inputs of the Hc x Wc node window at (x0, y0) of a 2D mesh with
 * nx x ny nodes, written to batch entry b: shared channels
 * (c, ratio (c_n - c_{n-1}), mu, ratio (mu_n - mu_{n-1})) scaled by scale[0..3],
 * grain channels (eta_i, ratio (eta_i,n - eta_i,n-1)) scaled by scale[4..5];
 * nodes outside the mesh read 0.  ratio = dt_n / dt_{n-1}. */
int sint_nn_features_f64(const double *u_n, const double *u_nm1, int64_t block_stride, int nx, int ny, int G, int x0,
                         int y0, int Hc, int Wc, float ratio, const float *scale, float *grain_in, float *shared_in,
                         int b, sint_stream_t stream);
/* Training targets of the same window: (u_{n+1} - u_n - ratio (u_n - u_{n-1}))
 * scaled by oscale[0] (c), oscale[1] (mu), oscale[2] (eta). */
int sint_nn_targets_f64(const double *u_np1, const double *u_n, const double *u_nm1, int64_t block_stride, int nx,
                        int ny, int G, int x0, int y0, int Hc, int Wc, float ratio, const float *oscale,
                        float *grain_t, float *shared_t, int b, sint_stream_t stream);
/* guess = u_n + ratio (u_n - u_{n-1}) + out / oscale over all n_nodes nodes
 * (network outputs of one whole-mesh window). */
int sint_nn_apply_guess_f64(const double *u_n, const double *u_nm1, int64_t block_stride, int64_t n_nodes, int G,
                            float ratio, const float *oscale, const float *grain_out, const float *shared_out,
                            double *guess, sint_stream_t stream);

/* 3D windows of D x H x W nodes at (x0, y0, z0) of an nx x ny x nz node mesh
 * (x fastest), held depth-major with a zero slice before and after:
 * grain_in [(b G + g)][D + 2][2][H][W], shared_in [b][D + 2][4][H][W];
 * the features of sint_nn_features_f64, written to slices 1 .. D (the zero
 * slices are left alone).  A 3x3x3 convolution of such a tensor is three 3x3
 * convolutions of its slice batch shifted by -1, 0, +1 slices. */
int sint_nn_features3d_f64(const double *u_n, const double *u_nm1, int64_t block_stride, int nx, int ny, int nz,
                           int G, int x0, int y0, int z0, int D, int H, int W, float ratio, const float *scale,
                           float *grain_in, float *shared_in, int b, sint_stream_t stream);
/* Training targets of a 3D window (layout grain_t [(b G + g)][D + 2][1][H][W],
 * shared_t [b][D + 2][2][H][W]), as sint_nn_targets_f64. */
int sint_nn_targets3d_f64(const double *u_np1, const double *u_n, const double *u_nm1, int64_t block_stride, int nx,
                          int ny, int nz, int G, int x0, int y0, int z0, int D, int H, int W, float ratio,
                          const float *oscale, float *grain_t, float *shared_t, int b, sint_stream_t stream);
/* guess = u_n + ratio (u_n - u_{n-1}) + out / oscale at the nodes of mesh
 * depth slices z0 .. z0 + D - 1, from the outputs of a whole-plane 3D window
 * (H = ny, W = nx) of Dw depth slices starting at mesh slice z0 - halo (its
 * padded slice 1 + halo + j holds mesh slice z0 + j). */
int sint_nn_apply_guess3d_f64(const double *u_n, const double *u_nm1, int64_t block_stride, int nx, int ny, int G,
                              int z0, int D, int halo, int Dw, float ratio, const float *oscale, const float *grain_out,
                              const float *shared_out, double *guess, sint_stream_t stream);
/* Zero depth slices 0 and D2 - 1 of each of S samples (slice_elems floats per
 * slice): the padding of a 3D window after a convolution wrote into it. */
int sint_nn_zero_pad_slices_f32(float *x, int S, int D2, int64_t slice_elems, sint_stream_t stream);
/* One-pass 3x3x3 convolution for inference on depth-padded windows
 * [S][D + 2][C][H][W] (slices 0 and D + 1 zero):
 *   out[s][z][co] = act(bias[co] + sum_{dz,dy,dx,ci} w1[dz][co][ci][dy][dx]
 *                   x1[s][z + dz - 1][ci][y + dy - 1][x + dx - 1] (+ the same for
 *                   x2, w2 with c2 channels) (+ addend[s / addend_group][z][co])
 *                   (+ out if accumulate)),
 * zero outside the window, for slices z = 1 .. D; slices 0 and D + 1 of out
 * are set to zero.  act = leaky ReLU with `slope` if leaky != 0.  FP32
 * products and sums; 1 <= cout <= 32; x2/w2 may be NULL (c2 = 0), so may
 * bias and addend (addend_group divides S). */
int sint_nn_conv3d_f32(int S, int D, int H, int W, const float *x1, int c1, const float *w1, const float *x2, int c2,
                       const float *w2, const float *bias, const float *addend, int addend_group, int leaky,
                       float slope, float *out, int cout, int accumulate, sint_stream_t stream);

/* Per-state scales of the network inputs and outputs: with m_c, m_mu, m_eta
 * the largest |ratio (u_n - u_{n-1})| of c, mu and any eta_i over the mesh and
 * dt the step being predicted, scale = (base[0], 1/m_c, base[1], 1/m_mu,
 * base[2], 1/m_eta) and oscale = (base[3], base[4], base[5]) / (m dt) per
 * group (device arrays; a zero increment gives 1/m = 1).  work: 3 device
 * unsigned ints of scratch. */
int sint_nn_increment_scales_f64(const double *u_n, const double *u_nm1, int64_t block_stride, int64_t n_nodes, int G,
                                 float ratio, float dt, const float *base, unsigned *work, float *scale,
                                 float *oscale, sint_stream_t stream);

/* Text of the last error recorded on this thread (never NULL). */
const char *sint_last_error(void);

/* Number of CUDA kernels this library has launched in this process. */
int64_t sint_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* HPSINT_B200_H */
