"""Host-side mirror of hpsint's sintering operator interface over the C ABI.

Class and method names follow the reference so that driver code reads the same:
  SinteringOperatorGeneric   applications/sintering/include/pf-applications/sintering/
                             operator_sintering_generic.h:323-1085
  BlockPreconditioner2       sintering/preconditioners.h:978-1343
  DampedNewtonSolver         include/pf-applications/lac/solvers_nonlinear.h:236-394
  bdf_weights                include/pf-applications/time_integration/time_schemes.h:64-153

Block vectors are torch CUDA tensors of shape (C, block_stride): torch only
provides device memory and the current stream; all arithmetic runs in the
library's CUDA kernels.
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L


@dataclass
class Mesh:
    """Uniform Cartesian mesh: n_cells cells of size h per direction."""
    dim: int
    n_cells: tuple
    h: tuple = (1.0, 1.0, 1.0)
    origin: tuple = (0.0, 0.0, 0.0)

    def to_c(self):
        m = L.SintMesh()
        m.dim = self.dim
        for d in range(3):
            m.n_cells[d] = int(self.n_cells[d]) if d < self.dim else 1
            m.h[d] = float(self.h[d]) if d < self.dim else 1.0
            m.origin[d] = float(self.origin[d]) if d < self.dim else 0.0
        return m

    @property
    def n_nodes(self):
        n = 1
        for d in range(self.dim):
            n *= int(self.n_cells[d]) + 1
        return n

    @property
    def node_shape(self):
        """(nz, ny, nx) node counts, the numpy shape of one block in C order."""
        s = [int(self.n_cells[d]) + 1 for d in range(self.dim)]
        return tuple(reversed(s))


@dataclass
class Params:
    """Model parameters; defaults are hpsint's EnergyAbstractData/MobilityAbstractData
    (sintering/parameters.h:113-134)."""
    n_grains: int
    A: float = 16.0
    B: float = 1.0
    kappa_c: float = 1.0
    kappa_p: float = 0.5
    Mvol: float = 1e-2
    Mvap: float = 1e-10
    Msurf: float = 4.0
    Mgb: float = 0.4
    L: float = 1.0
    tensorial: bool = True

    def to_c(self):
        return L.SintParams(self.n_grains, self.A, self.B, self.kappa_c, self.kappa_p, self.Mvol, self.Mvap,
                            self.Msurf, self.Mgb, self.L, int(bool(self.tensorial)))


def bdf_weights(order, dt):
    """BDF{1,2,3}Scheme::compute_weights (time_schemes.h:64-153) with the
    effective-order fallback; dt = [dt_n, dt_{n-1}, ...].  Returns w[0..order]."""
    dt = list(dt)
    eff = sum(1 for v in dt[:order] if v > 0)
    w = [0.0] * (len(dt) + 1)
    if eff >= 3 and order >= 3:
        w[1] = -(dt[0] + dt[1]) * (dt[0] + dt[1] + dt[2]) / (dt[0] * dt[1] * (dt[1] + dt[2]))
        w[2] = dt[0] * (dt[0] + dt[1] + dt[2]) / (dt[1] * dt[2] * (dt[0] + dt[1]))
        w[3] = -dt[0] * (dt[0] + dt[1]) / (dt[2] * (dt[1] + dt[2]) * (dt[0] + dt[1] + dt[2]))
        w[0] = -(w[1] + w[2] + w[3])
    elif eff >= 2 and order >= 2:
        w[0] = (2 * dt[0] + dt[1]) / (dt[0] * (dt[0] + dt[1]))
        w[1] = -(dt[0] + dt[1]) / (dt[0] * dt[1])
        w[2] = dt[0] / (dt[1] * (dt[0] + dt[1]))
    else:
        w[0] = 1.0 / dt[0]
        w[1] = -1.0 / dt[0]
    return w


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class SinteringOperatorGeneric:
    """Matrix-free sintering operator on the GPU (one CUDA context per instance)."""

    op_components_offset = 2

    def __init__(self, mesh: Mesh, params: Params):
        if not torch.cuda.is_available():
            raise RuntimeError("SinteringOperatorGeneric needs a CUDA device")
        self.mesh, self.params = mesh, params
        lib = L.lib()
        handle = ctypes.c_void_p()
        L.check(lib.sint_create(ctypes.byref(mesh.to_c()), ctypes.byref(params.to_c()), ctypes.byref(handle)),
                "sint_create")
        self._h = handle
        n, c, ld = ctypes.c_int64(), ctypes.c_int(), ctypes.c_int64()
        L.check(lib.sint_dof_layout(self._h, ctypes.byref(n), ctypes.byref(c), ctypes.byref(ld)), "sint_dof_layout")
        self.N, self.C, self.ld = n.value, c.value, ld.value
        self.order = 0
        self.cut_off_tolerance = 0.0

    @classmethod
    def create(cls, mesh, params):
        return cls(mesh, params)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib().sint_destroy(h)
            except Exception:
                pass
            self._h = None

    # --- reference interface ------------------------------------------------
    def n_components(self):
        return self.C

    def n_grains(self):
        return self.C - 2

    def equation_type(self, component):
        """operator_sintering_generic.h:634-639: mu is stationary."""
        return "Stationary" if component == 1 else "TimeDependent"

    def initialize_dof_vector(self, dtype=torch.float64):
        return torch.zeros((self.C, self.ld), dtype=dtype, device="cuda")

    def set_time_weights(self, w0, w_hist=(), w_alg=1.0):
        arr = (ctypes.c_double * max(1, len(w_hist)))(*w_hist)
        L.check(L.lib().sint_set_time_weights(self._h, float(w0), arr, len(w_hist), float(w_alg)),
                "sint_set_time_weights")
        self.order = len(w_hist)

    def set_mobility(self, Mvol, Mvap, Msurf, Mgb, L_):
        L.check(L.lib().sint_set_mobility(self._h, Mvol, Mvap, Msurf, Mgb, L_), "sint_set_mobility")

    def fill_quadrature_point_values(self, src):
        """Linearisation point (operator_sintering_data.h:300-409)."""
        self._check_vec(src, torch.float64)
        L.check(L.lib().sint_set_linearization_point(self._h, _ptr(src), _stream()), "sint_set_linearization_point")

    set_linearization_point = fill_quadrature_point_values

    def set_component_mask(self, src, grain_use_cut_off_tolerance):
        """Grain cut-off (SinteringOperatorData::set_component_mask,
        operator_sintering_data.h:149-298): grain b is relevant on a cell when
        max |eta_b| over the cell's nodes of `src` exceeds the tolerance; the
        residual and the Jacobian products then treat every cell with its
        relevant grains only (the preconditioner too after
        set_preconditioner_cut_off(True)).  Tolerance 0 switches the cut-off
        off (GrainCutOffTolerance, parameters.h:314)."""
        tol = float(grain_use_cut_off_tolerance)
        if tol != 0.0:
            self._check_vec(src, torch.float64)
        L.check(L.lib().sint_set_component_mask(self._h, _ptr(src) if tol != 0.0 else None, tol, _stream()),
                "sint_set_component_mask")
        self.cut_off_tolerance = tol

    def set_preconditioner_type(self, block_0):
        """Block 0 of the block preconditioner: "block_jacobi" (2x2 node
        blocks, default) or "ch_gauss_seidel" (the assembled Cahn-Hilliard
        block by multicolour symmetric Gauss-Seidel); takes effect at the next
        preconditioner set-up."""
        kind = BlockPreconditioner2.BLOCK0[block_0]
        L.check(L.lib().sint_set_preconditioner_type(self._h, kind), "sint_set_preconditioner_type")
        self.preconditioner_type = block_0

    def set_preconditioner_cut_off(self, on):
        """Build the block preconditioner with the grain cut-off too (the
        reference's assembly, preconditioners.h:787-817) instead of from the
        full operator (the default); takes effect at the next set-up."""
        L.check(L.lib().sint_set_preconditioner_cut_off(self._h, int(bool(on))), "sint_set_preconditioner_cut_off")

    def set_cut_off_skip_zero_chunks(self, on):
        """Under the cut-off the device GMRES skips the chunks of its vectors
        that are zero by construction (default on; results are bitwise the
        same either way)."""
        L.check(L.lib().sint_set_cut_off_skip_zero_chunks(self._h, int(bool(on))), "sint_set_cut_off_skip_zero_chunks")

    def cut_off_freeze(self, u, u_old):
        """u <- u_old on the DoFs the grain cut-off takes out of the system (a
        grain at a node none of whose cells has it relevant)."""
        self._check_vec(u, torch.float64)
        self._check_vec(u_old, torch.float64)
        L.check(L.lib().sint_cut_off_freeze(self._h, _ptr(u), _ptr(u_old), _stream()), "sint_cut_off_freeze")

    def component_mask_statistics(self):
        """numpy array: entry k = number of cells with k relevant grains
        (the "Cut-off statistic" of operator_sintering_data.h:236-296)."""
        counts = (ctypes.c_int64 * (self.params.n_grains + 1))()
        L.check(L.lib().sint_component_mask_statistics(self._h, counts, _stream()), "sint_component_mask_statistics")
        return np.array(counts[:], dtype=np.int64)

    def get_component_mask(self):
        """Device tensor of the cell masks (int16 bit patterns; bit b = grain b relevant), cells x-fastest."""
        n = 1
        for d in range(self.mesh.dim):
            n *= self.mesh.n_cells[d]
        out = torch.empty(n, dtype=torch.int16, device="cuda")
        L.check(L.lib().sint_get_component_mask(self._h, _ptr(out), _stream()), "sint_get_component_mask")
        return out

    def set_periodicity(self, directions):
        """Periodic directions (iterable of axis indices, e.g. (0, 1)); the
        nodes at the upper face become slaves of the lower face's
        (DoFTools::make_periodicity_constraints)."""
        bits = 0
        for d in directions:
            bits |= 1 << int(d)
        L.check(L.lib().sint_set_periodicity(self._h, bits), "sint_set_periodicity")
        self.periodic = tuple(sorted(int(d) for d in directions))

    def distribute_constraints(self, u):
        """Slave entries of u take their masters' values."""
        self._check_vec(u, torch.float64)
        L.check(L.lib().sint_distribute_constraints(self._h, _ptr(u), _stream()), "sint_distribute_constraints")

    def set_advection(self, cell_segments, segments):
        """Rigid-body motion of the grains (AdvectionMechanism,
        sintering/advection.h:297-520): the residual and J v gain the terms
        -(v_i c, grad phi) in the c row and -(v_i eta_i, grad phi) in the
        eta_i rows.  cell_segments: device int32 tensor (n_grains, n_cells),
        the segment of each order parameter a cell belongs to or -1;
        segments: device float64 tensor (n_segments, 9) = translational
        velocity, angular velocity (z only in 2D), center.  None switches
        advection off.  The tables are copied."""
        if cell_segments is None:
            L.check(L.lib().sint_set_advection(self._h, None, None, 0, _stream()), "sint_set_advection")
            return
        self._check_segments(cell_segments)
        if (segments.dtype != torch.float64 or not segments.is_cuda or not segments.is_contiguous()
                or segments.numel() % 9 != 0):
            raise ValueError("segments must be a contiguous float64 CUDA tensor of n_segments x 9 values")
        n_seg = segments.numel() // 9
        L.check(L.lib().sint_set_advection(self._h, _ptr(cell_segments), _ptr(segments) if n_seg else None, n_seg,
                                           _stream()), "sint_set_advection")

    def set_advection_mechanism(self, cell_segments, centers, k, cgb, ceq, smoothening, mt, mr):
        """The advection mechanism (AdvectionMechanism + AdvectionOperatorGeneric,
        sintering/advection.h, operator_advection.h): every residual evaluation
        first computes each segment's volume, force and torque from its state
        and moves the grain with v_t = mt F / V, w = mr T / V about its center;
        J v uses the velocities of the latest residual evaluation.
        cell_segments: device int32 (n_grains, n_cells), -1 = none; centers:
        device float64 (n_segments, 3).  None switches advection off."""
        if cell_segments is None:
            L.check(L.lib().sint_set_advection_mechanism(self._h, None, None, 0, None, _stream()),
                    "sint_set_advection_mechanism")
            return
        self._check_segments(cell_segments)
        if (centers.dtype != torch.float64 or not centers.is_cuda or not centers.is_contiguous()
                or centers.numel() % 3 != 0):
            raise ValueError("centers must be a contiguous float64 CUDA tensor of n_segments x 3 values")
        n_seg = centers.numel() // 3
        prm = L.SintAdvectionParams(float(k), float(cgb), float(ceq), float(smoothening), float(mt), float(mr))
        L.check(L.lib().sint_set_advection_mechanism(self._h, _ptr(cell_segments), _ptr(centers) if n_seg else None,
                                                     n_seg, ctypes.byref(prm), _stream()),
                "sint_set_advection_mechanism")
        self._n_segments = n_seg

    def advection_forces(self, u):
        """Volume, force and torque of every segment at state u (device
        float64 tensor (n_segments, 1 + dim + (3 or 1))); also updates the
        velocities J v uses."""
        self._check_vec(u, torch.float64)
        nc = 7 if self.mesh.dim == 3 else 4
        out = torch.zeros((getattr(self, "_n_segments", 0), nc), dtype=torch.float64, device="cuda")
        L.check(L.lib().sint_advection_forces(self._h, _ptr(u), _ptr(out) if out.numel() else None, _stream()),
                "sint_advection_forces")
        return out

    def check_courant(self, dt):
        """CFLChecker::check_courant with the current velocities: True when
        |v| dt < cell diameter everywhere a grain moves."""
        ok = ctypes.c_int()
        L.check(L.lib().sint_advection_check_courant(self._h, float(dt), ctypes.byref(ok), _stream()),
                "sint_advection_check_courant")
        return bool(ok.value)

    def _check_segments(self, cell_segments):
        n_cells = 1
        for d in range(self.mesh.dim):
            n_cells *= self.mesh.n_cells[d]
        if (cell_segments.dtype != torch.int32 or not cell_segments.is_cuda or not cell_segments.is_contiguous()
                or cell_segments.numel() != self.params.n_grains * n_cells):
            raise ValueError(f"cell_segments must be a contiguous int32 CUDA tensor of {self.params.n_grains} x "
                             f"{n_cells} ids")

    def evaluate_nonlinear_residual(self, dst, src, with_time_derivative=2, history=(), perturb=None,
                                    perturb_scale=0.0, subtract=None, scale=1.0):
        """dst = R(src) (operator_sintering_generic.h:393-448).  The range
        hooks of the reference's signature in device form: with `perturb`
        the residual is evaluated at src + perturb_scale * perturb (src is
        not modified), with `subtract` / `scale` it is stored as
        scale * (R - subtract) -- the pre/post operations of the
        Jacobian-free operator (lac/jacobian_operator.h:160-232), fused
        into the cell loop and its stores."""
        self._check_vec(dst, torch.float64)
        self._check_vec(src, torch.float64)
        hist = list(history)
        for h in hist:
            self._check_vec(h, torch.float64)
        arr = (ctypes.c_void_p * max(1, len(hist)))(*[h.data_ptr() for h in hist])
        if perturb is None and subtract is None and scale == 1.0:
            L.check(L.lib().sint_residual_f64(self._h, _ptr(dst), _ptr(src), arr, int(with_time_derivative),
                                              _stream()), "sint_residual_f64")
            return
        for v in (perturb, subtract):
            if v is not None:
                self._check_vec(v, torch.float64)
        hooks = L.SintResidualHooks(_ptr(perturb) if perturb is not None else None, float(perturb_scale),
                                    _ptr(subtract) if subtract is not None else None, float(scale))
        L.check(L.lib().sint_residual_f64_hooks(self._h, _ptr(dst), _ptr(src), arr, int(with_time_derivative),
                                                ctypes.byref(hooks), _stream()), "sint_residual_f64_hooks")

    def vmult(self, dst, src):
        if src.dtype == torch.float32:
            self._check_vec(dst, torch.float32)
            self._check_vec(src, torch.float32)
            L.check(L.lib().sint_jvp_f32(self._h, _ptr(dst), _ptr(src), _stream()), "sint_jvp_f32")
        else:
            self._check_vec(dst, torch.float64)
            self._check_vec(src, torch.float64)
            L.check(L.lib().sint_jvp_f64(self._h, _ptr(dst), _ptr(src), _stream()), "sint_jvp_f64")

    def do_update(self):
        pass

    def clear(self):
        pass

    def norm(self, v):
        """l2 norm of a whole FP64 block vector (deterministic device reduction); synchronises."""
        self._check_vec(v, torch.float64)
        out = torch.empty(1, dtype=torch.float64, device="cuda")
        L.check(L.lib().sint_vec_norm2_f64(self._h, v.numel(), _ptr(v), _ptr(out), _stream()), "sint_vec_norm2_f64")
        return float(out.item())

    # --- helpers --------------------------------------------------------------
    def _check_vec(self, t, dtype):
        if not (t.is_cuda and t.dtype == dtype and t.is_contiguous() and t.numel() == self.C * self.ld):
            raise ValueError(f"expected a contiguous CUDA {dtype} block vector of shape ({self.C}, {self.ld})")

    def to_device(self, arr_cn, dtype=torch.float64):
        """(C, N) array-like -> (C, ld) device block vector (padding zero)."""
        v = self.initialize_dof_vector(dtype)
        v[:, :self.N] = torch.as_tensor(arr_cn, dtype=dtype).reshape(self.C, self.N).to("cuda")
        return v

    def to_host(self, v):
        return v[:, :self.N].double().cpu().numpy()


class BlockPreconditioner2:
    """z = P^-1 r: the Cahn-Hilliard block by 2x2 node-block Jacobi
    (block_0="block_jacobi") or by a multicolour symmetric Gauss-Seidel sweep
    pair on the assembled Cahn-Hilliard matrix (block_0="ch_gauss_seidel",
    in place of the reference's ILU); the grains by their inverse diagonal.
    FP64 and FP32.  The block-0 type is a property of the operator context
    (the device Newton solver uses the same)."""

    BLOCK0 = {"block_jacobi": 0, "ch_gauss_seidel": 1}

    def __init__(self, op: SinteringOperatorGeneric, block_0=None):
        self.op = op
        if block_0 is not None:
            op.set_preconditioner_type(block_0)

    def do_update(self):
        L.check(L.lib().sint_precond_setup(self.op._h, _stream()), "sint_precond_setup")

    def vmult(self, dst, src):
        op = self.op
        if src.dtype == torch.float32:
            L.check(L.lib().sint_precond_apply_f32(op._h, _ptr(dst), _ptr(src), _stream()), "sint_precond_apply_f32")
        else:
            L.check(L.lib().sint_precond_apply_f64(op._h, _ptr(dst), _ptr(src), _stream()), "sint_precond_apply_f64")

    def inverse_diagonal(self):
        G = self.op.n_grains()
        out = torch.zeros((G, self.op.ld), dtype=torch.float64, device="cuda")
        L.check(L.lib().sint_ac_inverse_diagonal_f64(self.op._h, _ptr(out), _stream()), "sint_ac_inverse_diagonal_f64")
        return out

    def ch_blocks(self):
        out = torch.zeros((4, self.op.ld), dtype=torch.float64, device="cuda")
        L.check(L.lib().sint_ch_blocks_f64(self.op._h, _ptr(out), _stream()), "sint_ch_blocks_f64")
        return out

    def ch_matrix(self):
        """The assembled Cahn-Hilliard block (block_0="ch_gauss_seidel"):
        (3^dim, 4, ld) = 2x2 blocks per node row and neighbour."""
        nk = 27 if self.op.mesh.dim == 3 else 9
        out = torch.zeros((nk, 4, self.op.ld), dtype=torch.float64, device="cuda")
        L.check(L.lib().sint_ch_matrix_f64(self.op._h, _ptr(out), _stream()), "sint_ch_matrix_f64")
        return out

    def clear(self):
        pass


@dataclass
class NonLinearData:
    """lac/solvers_nonlinear_parameters.h:40-60 (+ GMRES restart and inner precision)."""
    nl_max_iter: int = 10
    nl_abs_tol: float = 1e-20
    nl_rel_tol: float = 1e-5
    l_max_iter: int = 1000
    l_abs_tol: float = 1e-10
    l_rel_tol: float = 1e-2
    gmres_restart: int = 30
    threshold_newton_iter: int = 100
    threshold_linear_iter: int = 20
    use_damping: bool = True
    reuse_preconditioner: bool = True
    inner_precision: int = 64
    right_preconditioning: bool = False

    def to_c(self):
        return L.SintNewtonParams(self.nl_max_iter, self.nl_abs_tol, self.nl_rel_tol, self.l_max_iter,
                                  self.l_abs_tol, self.l_rel_tol, self.gmres_restart, self.threshold_newton_iter,
                                  self.threshold_linear_iter, int(self.use_damping), int(self.reuse_preconditioner),
                                  self.inner_precision, int(self.right_preconditioning))


@dataclass
class NewtonStatistics:
    newton_iterations: int = 0
    linear_iterations: int = 0
    residual_evaluations: int = 0
    jacobian_setups: int = 0
    preconditioner_setups: int = 0
    initial_residual: float = 0.0
    final_residual: float = 0.0
    status: int = 0


class DampedNewtonSolver:
    """Device damped Newton-GMRES for R(u) = 0 (time weights set on the operator)."""

    def __init__(self, op: SinteringOperatorGeneric, data: NonLinearData = None):
        self.op = op
        self.data = data or NonLinearData()

    def solve(self, u, history, raise_on_failure=True, data: NonLinearData = None):
        """data overrides the solver's NonLinearData for this solve only."""
        op = self.op
        op._check_vec(u, torch.float64)
        arr = (ctypes.c_void_p * max(1, len(history)))(*[h.data_ptr() for h in history])
        st = L.SintNewtonStats()
        prm = (data or self.data).to_c()
        rc = L.lib().sint_newton_solve(op._h, _ptr(u), arr, ctypes.byref(prm), ctypes.byref(st), _stream())
        stats = NewtonStatistics(st.newton_iterations, st.linear_iterations, st.residual_evaluations,
                                 st.jacobian_setups, st.preconditioner_setups, st.initial_residual,
                                 st.final_residual, rc)
        if rc != L.SINT_OK and raise_on_failure:
            L.check(rc, "sint_newton_solve")
        return stats

    def clear(self):
        L.check(L.lib().sint_newton_clear(self.op._h), "sint_newton_clear")


class HostJvpPipeline:
    """J(u) v for vectors that live in (pinned) host memory, pipelined.

    A caller whose vectors stay on the host (a CPU driver handing one vector
    at a time to the GPU operator) pays a host-to-device copy, the product
    and a device-to-host copy per call.  Here consecutive calls overlap: the
    copy-in of call k + 1, the product of call k and the copy-out of call
    k - 1 run on three streams with double-buffered device vectors, so the
    throughput is set by the slowest of the three instead of their sum.
    `submit` returns at once; `synchronize` waits for every submitted call.
    Host buffers must be pinned (torch pin_memory) and stay untouched until
    their call is synchronised.
    """

    def __init__(self, op: SinteringOperatorGeneric, depth=2):
        if depth < 1:
            raise ValueError("depth must be >= 1")
        self.op = op
        self.depth = depth
        self.src = [op.initialize_dof_vector() for _ in range(depth)]
        self.dst = [op.initialize_dof_vector() for _ in range(depth)]
        self.s_in, self.s_jv, self.s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
        self.copied_in = [torch.cuda.Event() for _ in range(depth)]
        self.computed = [torch.cuda.Event() for _ in range(depth)]
        self.copied_out = [torch.cuda.Event() for _ in range(depth)]
        self.k = 0
        self.launched = [False] * depth
        self.begin()

    def submit(self, dst_host, src_host):
        """Queue dst_host = J src_host (both pinned (C, block_stride) float64 CPU tensors)."""
        i = self.k % self.depth
        op = self.op
        with torch.cuda.stream(self.s_in):
            if self.launched[i]:
                self.s_in.wait_event(self.computed[i])      # the product has read src[i]
            self.src[i].copy_(src_host, non_blocking=True)
            self.copied_in[i].record(self.s_in)
        with torch.cuda.stream(self.s_jv):
            self.s_jv.wait_event(self.copied_in[i])
            if self.launched[i]:
                self.s_jv.wait_event(self.copied_out[i])    # dst[i] was copied out
            L.check(L.lib().sint_jvp_f64(op._h, _ptr(self.dst[i]), _ptr(self.src[i]),
                                         ctypes.c_void_p(self.s_jv.cuda_stream)), "sint_jvp_f64")
            self.computed[i].record(self.s_jv)
        with torch.cuda.stream(self.s_out):
            self.s_out.wait_event(self.computed[i])
            dst_host.copy_(self.dst[i], non_blocking=True)
            self.copied_out[i].record(self.s_out)
        self.launched[i] = True
        self.k += 1

    def begin(self, stream=None):
        """Order the pipeline after everything queued so far on `stream` (default: current)."""
        ev = torch.cuda.Event()
        ev.record(stream or torch.cuda.current_stream())
        for s in (self.s_in, self.s_jv, self.s_out):
            s.wait_event(ev)

    def end(self, stream=None):
        """Make `stream` (default: current) wait for every submitted call."""
        stream = stream or torch.cuda.current_stream()
        for s in (self.s_in, self.s_jv, self.s_out):
            ev = torch.cuda.Event()
            ev.record(s)
            stream.wait_event(ev)

    def synchronize(self):
        for s in (self.s_in, self.s_jv, self.s_out):
            s.synchronize()
