"""Learned Newton initial guess: data, training, predictors and evaluation.

The workload is the 2D packing of many grains: Q1 on an n x n cell mesh at
unit spacing, circles with radii U[rmin, rmax] packed so that neighbours
overlap by 2 cells, greedily coloured to at most 8 order parameters.  The
FP64 device solver generates trajectories (every accepted state stays in HBM
as an FP64 block vector); the network (predictor.EquivariantNet) is trained
on random windows of (u_{n-1}, u_n, dt_{n-1}, dt_n -> u_{n+1}) triples with
the library's own forward/backward/Adam kernels; the trained net then plugs
into TimeIntegrator's predictor hook (hpsint's predictor switch,
sintering/driver.h:2001-2058).  hpsint's "Linear" predictor
(solution_history.h extrapolate with fac = dt_n / dt_{n-1}) is provided as
LinearPredictor, the thing the network improves on.

Nothing here decides the answer: each step is still the damped
Newton-Krylov solve to the same tolerance.
"""
import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from . import packings as PK
from .operator import Mesh, NonLinearData, Params, SinteringOperatorGeneric
from .predictor import EquivariantNet, NetConfig
from .time_integration import TimeIntegrationData, TimeIntegrator


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _s():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


# --- workload ------------------------------------------------------------------

def packing_2d(seed, n=512, n_circles=100, rmin=6.0, rmax=12.0, overlap=2.0, max_grains=8):
    """Seeded circle packing on [0, n]^2 coloured to <= max_grains order
    parameters: the colouring buffer (distance between surfaces below which
    two grains get different colours) is the largest of 32, 28, ..., 4 cells
    whose greedy colouring fits, so grains sharing an order parameter stay as
    far apart as the budget allows."""
    rng = np.random.default_rng(seed)
    centers, radii = PK.place_spheres(2, [0.0, 0.0], [float(n), float(n)], n_circles,
                                      lambda r: r.uniform(rmin, rmax), overlap, rng)
    for buffer in (32.0, 28.0, 24.0, 20.0, 16.0, 12.0, 8.0, 4.0):
        colours = PK.greedy_colouring(centers, radii, buffer)
        if colours.max() + 1 <= max_grains:
            return centers, radii, colours
    raise RuntimeError(f"packing seed {seed}: no colouring with <= {max_grains} order parameters")


def model_params(G, tensorial=False):
    """hpsint's default energy and mobility constants.  Scalar mobility by
    default: the tensorial tangent is inexact in hpsint (its tangent tester
    accepts a looser bound for it, tangent_tester.h), and over long runs
    Newton stalls near 1e-4 relative with it, so FP64 trajectories to the
    1e-8 tolerance need dt halvings down to the minimum; with the scalar
    mobility the tangent is exact and every step converges."""
    return Params(n_grains=G, A=16.0, B=1.0, kappa_c=1.0, kappa_p=0.5, Mvol=1e-2, Mvap=1e-10, Msurf=4.0,
                  Mgb=0.4, L=1.0, tensorial=tensorial)


@dataclass
class Case:
    """One packing: its operator and initial state (device)."""
    seed: int
    n: int
    G: int
    op: SinteringOperatorGeneric
    u0: torch.Tensor

    @property
    def nodes(self):
        return self.n + 1


def make_case(seed, n=512, n_circles=100, rmin=6.0, rmax=12.0, tensorial=False):
    centers, radii, colours = packing_2d(seed, n, n_circles, rmin, rmax)
    G = int(colours.max()) + 1
    u0 = PK.initial_state(2, (n, n), (1.0, 1.0), (0.0, 0.0), centers, radii, colours, width=2.0)
    op = SinteringOperatorGeneric(Mesh(2, (n, n, 1)), model_params(G, tensorial))
    return Case(seed, n, G, op, op.to_device(u0))


# --- trajectories -----------------------------------------------------------------

@dataclass
class Trajectory:
    """Accepted states u_0..u_K (FP64 device block vectors) and dts[k] = t_{k+1} - t_k."""
    case: Case
    states: list
    dts: list
    records: list = field(default_factory=list)

    def n_triples(self):
        return max(0, len(self.states) - 2)


def generate_trajectory(case, n_steps, nl=None, td=None):
    """FP64 device solve (hpsint's dt control, previous-solution guess) that keeps every state."""
    nl = nl or NonLinearData(nl_rel_tol=1e-8)
    td = td or TimeIntegrationData(time_step_init=1e-3)
    ti = TimeIntegrator(case.op, nl, td)
    ti.initialize(case.u0)
    _, states = ti.run(n_steps, keep_states=True)
    return Trajectory(case, states, [r.dt for r in ti.records], ti.records)


# --- normalisation -----------------------------------------------------------------

@dataclass
class Normaliser:
    """Scales of the network's inputs and outputs.  Per state, m_c, m_mu and
    m_eta are the largest extrapolated increments |r (u_n - u_{n-1})| of c,
    mu and the eta_i over the mesh (computed on the device); the increments
    enter divided by them, the values c, mu, eta times the fixed base scales.
    The output is the deviation from linear extrapolation divided by m dt_n
    (dt_n the predicted step) times the fixed gains: for a smooth trajectory
    that deviation is about dt_n J(u) r (u_n - u_{n-1}), so the scaled target
    depends on the state and the normalised increment only.  base = (s_c,
    s_mu, s_eta, k_c, k_mu, k_eta): s the reciprocal RMS of the values, k the
    reciprocal RMS of deviation / (m dt) over the training triples."""
    base: list

    def device(self):
        return torch.tensor(self.base, dtype=torch.float32, device="cuda")


class IncrementScales:
    """Device scale (6 floats) and oscale (3 floats) of one state via
    sint_nn_increment_scales_f64."""

    def __init__(self):
        self.work = torch.zeros(4, dtype=torch.int32, device="cuda")

    def __call__(self, un, um, ld, n_nodes, G, ratio, dt, base, scale, oscale):
        L.check(L.lib().sint_nn_increment_scales_f64(_p(un), _p(um), ld, n_nodes, G, ratio, dt, _p(base),
                                                     _p(self.work), _p(scale), _p(oscale), _s()),
                "sint_nn_increment_scales_f64")


def _triple_scales(tr, base, inc):
    """(scales [K][6], oscales [K][3]) of every triple centre k = 1..K-1 (row k)."""
    K = len(tr.states)
    sc = torch.ones((K, 6), dtype=torch.float32, device="cuda")
    osc = torch.ones((K, 3), dtype=torch.float32, device="cuda")
    for k in range(1, K - 1):
        inc(tr.states[k], tr.states[k - 1], tr.case.op.ld, tr.case.op.N, tr.case.G, tr.dts[k] / tr.dts[k - 1],
            tr.dts[k], base, sc[k], osc[k])
    return sc, osc


def fit_normaliser(trajs, max_triples=400):
    """base scales from the training trajectories (statistics via torch on the device)."""
    ones = torch.ones(6, dtype=torch.float32, device="cuda")
    inc = IncrementScales()
    vsum, dsum, cnt = np.zeros(3), np.zeros(3), np.zeros(3)
    used = 0
    for tr in trajs:
        G, N = tr.case.G, tr.case.op.N
        sc, _ = _triple_scales(tr, ones, inc)
        inv_m = sc[:, 1::2].double().cpu().numpy()  # 1 / m per triple
        for k in range(1, len(tr.states) - 1):
            if used >= max_triples:
                break
            r = tr.dts[k] / tr.dts[k - 1]
            un, um, up = (tr.states[j][:, :N] for j in (k, k - 1, k + 1))
            dev = up - un - r * (un - um)
            for g, (i0, i1) in enumerate(((0, 1), (1, 2), (2, 2 + G))):
                vsum[g] += float((un[i0:i1] ** 2).sum())
                dsum[g] += float((dev[i0:i1] ** 2).sum()) * (inv_m[k, g] / tr.dts[k]) ** 2
                cnt[g] += (i1 - i0) * N
            used += 1
    cnt = np.maximum(cnt, 1)
    inv = lambda x: float(1.0 / x) if x > 1e-30 else 1.0
    s = [inv(np.sqrt(v)) for v in vsum / cnt]
    k = [inv(np.sqrt(d)) for d in dsum / cnt]
    return Normaliser(s + k)


# --- training ----------------------------------------------------------------------

@dataclass
class TrainConfig:
    window: int = 64          # Hc = Wc nodes per training window
    batch: int = 16           # windows per Adam step (all from one trajectory: same G)
    iterations: int = 2000
    lr: float = 1e-3
    lr_final: float = 1e-5    # cosine decay from lr to lr_final over the iterations (lr_final = lr: constant)
    seed: int = 0
    log_every: int = 100
    # weight of the curvature term: mean of (5-point Laplacian of the masked
    # error)^2, which penalises the high-frequency error the fourth-order
    # Cahn-Hilliard operator amplifies in the Newton residual (0: plain MSE)
    smooth: float = 4.0


class WindowSampler:
    """Random windows of random triples.  Window origins are drawn where the
    window holds some material (max c > 0.01 over a stride-16 grid of
    candidate origins, found once per trajectory on the host) and may reach
    `margin` nodes past the mesh, where the features read zero, the padding
    the whole-mesh inference sees."""

    def __init__(self, trajs, window, margin, rng):
        self.trajs = [t for t in trajs if t.n_triples() > 0]
        if not self.trajs:
            raise ValueError("no trajectory with at least one (u_{n-1}, u_n, u_{n+1}) triple")
        self.window, self.margin, self.rng = window, margin, rng
        self.origins = []
        for tr in self.trajs:
            nn = tr.case.nodes
            c = tr.states[0][0, :tr.case.op.N].view(nn, nn).cpu().numpy()
            cand = []
            lo, hi = -margin, nn - window + margin
            for y0 in range(lo, max(lo, hi) + 1, 16):
                for x0 in range(lo, max(lo, hi) + 1, 16):
                    ys, xs = max(0, y0), max(0, x0)
                    if c[ys:y0 + window, xs:x0 + window].max(initial=0.0) > 0.01:
                        cand.append((x0, y0))
            self.origins.append(cand or [(lo, lo)])

    def draw(self):
        """(trajectory, [(k, x0, y0) per window])."""
        ti = int(self.rng.integers(len(self.trajs)))
        tr, cand = self.trajs[ti], self.origins[ti]
        out = []
        for _ in range(self.batch_size):
            k = int(self.rng.integers(1, len(tr.states) - 1))
            x0, y0 = cand[int(self.rng.integers(len(cand)))]
            jx, jy = self.rng.integers(-8, 9, size=2)
            hi = tr.case.nodes - self.window + self.margin
            x0 = int(min(max(x0 + jx, -self.margin), hi))
            y0 = int(min(max(y0 + jy, -self.margin), hi))
            out.append((k, x0, y0))
        return tr, out


class Trainer:
    """Adam on the border-masked MSE between network output and the scaled
    deviation of u_{n+1} from linear extrapolation.  The mask drops a ring of
    `layers` nodes at the window edge (their receptive field leaves the
    window) and nodes outside the mesh."""

    def __init__(self, net: EquivariantNet, norm: Normaliser, trajs, cfg: TrainConfig = None):
        self.net, self.norm, self.cfg = net, norm, cfg or TrainConfig()
        self.rng = np.random.default_rng(self.cfg.seed)
        self.margin = net.cfg.layers
        self.sampler = WindowSampler(trajs, self.cfg.window, self.margin, self.rng)
        self.sampler.batch_size = self.cfg.batch
        base, inc = norm.device(), IncrementScales()
        self.scales = {id(tr): _triple_scales(tr, base, inc) for tr in self.sampler.trajs}
        self.history = []
        self._bufs = {}

    def _buffers(self, G):
        if G not in self._bufs:
            B, Wn = self.cfg.batch, self.cfg.window
            f = lambda *s: torch.zeros(s, dtype=torch.float32, device="cuda")
            self._bufs[G] = dict(xg=f(B * G, 2, Wn, Wn), xs=f(B, 4, Wn, Wn), tg=f(B * G, 1, Wn, Wn),
                                 ts=f(B, 2, Wn, Wn), wg=f(B * G, 1, Wn, Wn), ws=f(B, 2, Wn, Wn),
                                 dyg=f(B * G, 1, Wn, Wn), dys=f(B, 2, Wn, Wn))
        return self._bufs[G]

    def _window_mask(self, x0, y0, nodes):
        Wn, m = self.cfg.window, self.margin
        mask = torch.zeros((Wn, Wn), dtype=torch.float32, device="cuda")
        ylo, yhi = max(m, -y0), min(Wn - m, nodes - y0)
        xlo, xhi = max(m, -x0), min(Wn - m, nodes - x0)
        if ylo < yhi and xlo < xhi:
            mask[ylo:yhi, xlo:xhi] = 1.0
        return mask

    def fill_batch(self):
        tr, picks = self.sampler.draw()
        G, nodes, ld = tr.case.G, tr.case.nodes, tr.case.op.ld
        b = self._buffers(G)
        Wn = self.cfg.window
        lib = L.lib()
        sc, osc = self.scales[id(tr)]
        for i, (k, x0, y0) in enumerate(picks):
            un, um, up = tr.states[k], tr.states[k - 1], tr.states[k + 1]
            r = tr.dts[k] / tr.dts[k - 1]
            L.check(lib.sint_nn_features_f64(_p(un), _p(um), ld, nodes, nodes, G, x0, y0, Wn, Wn, r, _p(sc[k]),
                                             _p(b["xg"]), _p(b["xs"]), i, _s()), "sint_nn_features_f64")
            L.check(lib.sint_nn_targets_f64(_p(up), _p(un), _p(um), ld, nodes, nodes, G, x0, y0, Wn, Wn, r,
                                            _p(osc[k]), _p(b["tg"]), _p(b["ts"]), i, _s()),
                    "sint_nn_targets_f64")
            mask = self._window_mask(x0, y0, nodes)
            b["wg"][i * G:(i + 1) * G, 0].copy_(mask.expand(G, Wn, Wn))
            b["ws"][i, :].copy_(mask.expand(2, Wn, Wn))
        return G, b

    def lr_at(self, it, n):
        c = self.cfg
        return c.lr_final + 0.5 * (c.lr - c.lr_final) * (1.0 + math.cos(math.pi * min(it, n) / max(n, 1)))

    def _smooth_term(self, pred, target, weight, grad):
        """lambda mean((Delta (w (pred - target)))^2); adds lambda 2/n w Delta(Delta(w e)) to grad
        (grad may be None).  Delta: 5-point Laplacian with zero padding (a symmetric stencil, so
        its transpose is itself), applied per channel by the FP32 conv kernel."""
        from . import predictor as P
        lam = self.cfg.smooth
        H, W = pred.shape[-2], pred.shape[-1]
        e = torch.empty_like(pred)
        L.check(L.lib().sint_nn_weighted_diff_f32(pred.numel(), _p(pred), _p(target), _p(weight), _p(e), _s()),
                "sint_nn_weighted_diff_f32")
        lap = torch.empty_like(pred)
        P.conv3x3(e.view(-1, 1, H, W), self._lap, None, lap.view(-1, 1, H, W))
        g_l = torch.empty_like(pred) if grad is not None else None
        loss = self.net.mse(lap, torch.zeros_like(lap), None, g_l)
        if grad is not None:
            q = torch.empty_like(pred)
            P.conv3x3(g_l.view(-1, 1, H, W), self._lap, None, q.view(-1, 1, H, W))
            L.check(L.lib().sint_nn_mul_add_f32(pred.numel(), lam, _p(weight), _p(q), _p(grad), _s()),
                    "sint_nn_mul_add_f32")
        return loss * lam

    def step(self, lr=None):
        """One Adam step; returns (batch loss, loss of predicting zero = linear
        extrapolation) as device scalars (no sync)."""
        G, b = self.fill_batch()
        B = self.cfg.batch
        yg, ys, cache = self.net.forward(b["xg"], b["xs"], B, G, keep=True)
        lg = self.net.mse(yg, b["tg"], b["wg"], b["dyg"])
        ls = self.net.mse(ys, b["ts"], b["ws"], b["dys"])
        zg, zs = torch.zeros_like(b["tg"]), torch.zeros_like(b["ts"])
        base = self.net.mse(zg, b["tg"], b["wg"], None) + self.net.mse(zs, b["ts"], b["ws"], None)
        if self.cfg.smooth > 0:
            if not hasattr(self, "_lap"):
                self._lap = torch.tensor([[0.0, 1.0, 0.0], [1.0, -4.0, 1.0], [0.0, 1.0, 0.0]], dtype=torch.float32,
                                         device="cuda").view(1, 1, 3, 3)
            lg = lg + self._smooth_term(yg, b["tg"], b["wg"], b["dyg"])
            ls = ls + self._smooth_term(ys, b["ts"], b["ws"], b["dys"])
            base = base + self._smooth_term(zg, b["tg"], b["wg"], None) + self._smooth_term(zs, b["ts"], b["ws"], None)
        self.net.zero_grad()
        self.net.backward(cache, b["dyg"], b["dys"], B, G)
        self.net.adam_step(lr=self.cfg.lr if lr is None else lr)
        return lg + ls, base

    def train(self, iterations=None, verbose=False):
        n = iterations if iterations is not None else self.cfg.iterations
        t0 = time.perf_counter()
        acc, accb, cnt = None, None, 0
        for it in range(1, n + 1):
            loss, base = self.step(self.lr_at(it - 1, n))
            acc = loss if acc is None else acc + loss
            accb = base if accb is None else accb + base
            cnt += 1
            if it % self.cfg.log_every == 0 or it == n:
                mean, mb = float(acc.item()) / cnt, float(accb.item()) / cnt
                self.history.append((it, mean, mb))
                if verbose:
                    print(f"iter {it:6d}  loss {mean:.4e}  (zero prediction {mb:.4e})  "
                          f"{time.perf_counter() - t0:.1f}s", flush=True)
                acc, accb, cnt = None, None, 0
        torch.cuda.synchronize()
        return time.perf_counter() - t0


# --- predictors (TimeIntegrator hook) -------------------------------------------------

class LinearPredictor:
    """hpsint's "Linear" predictor: u_n + r (u_n - u_{n-1}), r = dt_n / dt_{n-1}
    (driver.h:2024-2036, SolutionHistory::extrapolate).  First step: None."""

    def __init__(self, op: SinteringOperatorGeneric):
        self.op = op
        self.guess = None

    def __call__(self, history, dts, dt):
        if len(history) < 2 or not dts or dts[0] <= 0:
            return None
        if self.guess is None:
            self.guess = self.op.initialize_dof_vector()
        r = dt / dts[0]
        self.guess.copy_(history[0])
        L.check(L.lib().sint_vec_sadd_f64(self.guess.numel(), 1.0 + r, -r, _p(history[1]), _p(self.guess), _s()),
                "sint_vec_sadd_f64")
        return self.guess


class EulerPredictor:
    """hpsint's "Euler" predictor (driver.h:2005-2011): the residual without
    time terms R0(u_n) (evaluate_nonlinear_residual<0>), then
    extrap = u_n - dt R0(u_n) (VectorType::sadd).  As in the reference it
    acts from the second step on (t > 0)."""

    def __init__(self, op: SinteringOperatorGeneric):
        self.op = op
        self.guess = None

    def _euler(self, out, u, dt):
        self.op.evaluate_nonlinear_residual(out, u, 0)
        L.check(L.lib().sint_vec_sadd_f64(out.numel(), -dt, 1.0, _p(u), _p(out), _s()), "sint_vec_sadd_f64")

    def __call__(self, history, dts, dt):
        if len(history) < 2 or not dts:
            return None
        if self.guess is None:
            self.guess = self.op.initialize_dof_vector()
        self._euler(self.guess, history[0], dt)
        return self.guess


class MidpointPredictor(EulerPredictor):
    """hpsint's "Midpoint" predictor (driver.h:2012-2023): midpoint =
    u_n - dt/2 R0(u_n), extrap = u_n - dt R0(midpoint)."""

    def __init__(self, op: SinteringOperatorGeneric):
        super().__init__(op)
        self.mid = None

    def __call__(self, history, dts, dt):
        if len(history) < 2 or not dts:
            return None
        if self.guess is None:
            self.guess, self.mid = self.op.initialize_dof_vector(), self.op.initialize_dof_vector()
        self._euler(self.mid, history[0], dt / 2.0)
        self.op.evaluate_nonlinear_residual(self.guess, self.mid, 0)
        L.check(L.lib().sint_vec_sadd_f64(self.guess.numel(), -dt, 1.0, _p(history[0]), _p(self.guess), _s()),
                "sint_vec_sadd_f64")
        return self.guess


class LearnedPredictor:
    """Whole-mesh inference: features of (u_{n-1}, u_n, r) -> net -> guess
    u_n + r (u_n - u_{n-1}) + output / oscale.  FP32 network, FP64 guess.

    safeguard: also form the linear guess, evaluate the residual of both
    under the step's time weights (set by the integrator before it asks for
    a guess) and keep the smaller, all on the device (no host sync), so the
    guess is never worse than hpsint's linear predictor in residual norm."""

    def __init__(self, op: SinteringOperatorGeneric, net: EquivariantNet, norm: Normaliser, tensor_cores=True,
                 safeguard=False):
        self.op, self.net, self.tensor_cores, self.safeguard = op, net, tensor_cores, safeguard
        self.base, self.inc = norm.device(), IncrementScales()
        self.scale = torch.ones(6, dtype=torch.float32, device="cuda")
        self.oscale = torch.ones(3, dtype=torch.float32, device="cuda")
        if op.mesh.dim != 2:
            raise ValueError("the learned predictor runs on 2D meshes")
        self.nx, self.ny = op.mesh.n_cells[0] + 1, op.mesh.n_cells[1] + 1
        G = op.params.n_grains
        f = lambda *s: torch.zeros(s, dtype=torch.float32, device="cuda")
        self.xg, self.xs = f(G, 2, self.ny, self.nx), f(1, 4, self.ny, self.nx)
        self.guess = op.initialize_dof_vector()
        self.calls = 0
        if safeguard:
            self.linear = LinearPredictor(op)
            self.r = op.initialize_dof_vector()
            self.norms = torch.zeros(2, dtype=torch.float64, device="cuda")
            self.picked_linear = torch.zeros(1, dtype=torch.float64, device="cuda")

    def __call__(self, history, dts, dt):
        if len(history) < 2 or not dts or dts[0] <= 0:
            return None
        op, G = self.op, self.op.params.n_grains
        r = dt / dts[0]
        lib = L.lib()
        self.inc(history[0], history[1], op.ld, op.N, G, r, dt, self.base, self.scale, self.oscale)
        L.check(lib.sint_nn_features_f64(_p(history[0]), _p(history[1]), op.ld, self.nx, self.ny, G, 0, 0, self.ny,
                                         self.nx, r, _p(self.scale), _p(self.xg), _p(self.xs), 0, _s()),
                "sint_nn_features_f64")
        yg, ys, _ = self.net.forward(self.xg, self.xs, 1, G, tensor_cores=self.tensor_cores)
        L.check(lib.sint_nn_apply_guess_f64(_p(history[0]), _p(history[1]), op.ld, op.N, G, r, _p(self.oscale),
                                            _p(yg), _p(ys), _p(self.guess), _s()), "sint_nn_apply_guess_f64")
        self.calls += 1
        if self.safeguard:
            lin = self.linear(history, dts, dt)
            n = self.guess.numel()
            for i, g in enumerate((self.guess, lin)):
                op.evaluate_nonlinear_residual(self.r, g, 2, history[:max(1, op.order)])
                L.check(lib.sint_vec_norm2_f64(op._h, n, _p(self.r), _p(self.norms[i:]), _s()), "sint_vec_norm2_f64")
            L.check(lib.sint_vec_select_f64(n, _p(self.guess), _p(lin), _p(self.norms[0:]), _p(self.norms[1:]),
                                            _p(self.guess), _s()), "sint_vec_select_f64")
            self.picked_linear += (self.norms[1] < self.norms[0]).double()
        return self.guess


# --- evaluation -------------------------------------------------------------------------

GRAIN_CUT_OFF = 1e-5  # GrainCutOffTolerance of the *_cut_off arms

ARMS = {
    # label: (inner precision, predictor, grain cut-off tolerance)
    "fp64_plain": (64, None, 0.0),
    "fp64_linear": (64, "linear", 0.0),
    "fp64_learned": (64, "learned", 0.0),
    "fp64_learned_safeguarded": (64, "learned_safeguarded", 0.0),
    "fp32_inner_plain": (32, None, 0.0),
    "fp32_inner_linear": (32, "linear", 0.0),
    "fp64_euler": (64, "euler", 0.0),
    "fp64_midpoint": (64, "midpoint", 0.0),
    "fp32_inner_euler": (32, "euler", 0.0),
    "fp32_inner_midpoint": (32, "midpoint", 0.0),
    "fp32_inner_learned": (32, "learned", 0.0),
    "fp32_inner_learned_safeguarded": (32, "learned_safeguarded", 0.0),
    "fp32_inner_linear_cut_off": (32, "linear", GRAIN_CUT_OFF),
    "fp32_inner_learned_safeguarded_cut_off": (32, "learned_safeguarded", GRAIN_CUT_OFF),
}


def lumped_mass_2d(nodes):
    w = np.ones(nodes)
    w[[0, -1]] = 0.5
    return np.outer(w, w).ravel()


def run_arm(case, n_steps, inner_precision, predictor, dt_schedule=None, nl_rel_tol=1e-8, cut_off=0.0):
    """One solve of n_steps from case.u0 (with the grain cut-off when
    cut_off > 0); returns (final state on the host, records, wall seconds)."""
    nl = NonLinearData(nl_rel_tol=nl_rel_tol, inner_precision=inner_precision)
    case.op.set_component_mask(case.u0, cut_off)  # 0: switch a previous arm's cut-off off
    ti = TimeIntegrator(case.op, nl, TimeIntegrationData(time_step_init=1e-3), predictor=predictor,
                        tolerance_base="old_solution", grain_cut_off_tolerance=cut_off)
    ti.initialize(case.u0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ti.run(n_steps, dt_schedule=dt_schedule)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    return case.op.to_host(ti.history[0]), ti.records, wall


def _gmean(x):
    return float(np.exp(np.mean(np.log(x)))) if len(x) else None


def compare_arms(case, n_steps, net=None, norm=None, arms=None, warmup_steps=2):
    """Runs the arms on the same packing.  fp64_plain (hpsint's method: FP64,
    previous-solution guess, adaptive dt) runs first and fixes the time grid;
    every other arm replays its dt schedule so final fields compare on the same
    grid.  Reports per arm s/step, Newton/GMRES iterations and the max-norm
    difference of c and eta from fp64_plain at the final step."""
    arms = list(arms or ARMS)
    if arms[0] != "fp64_plain":
        arms = ["fp64_plain"] + [a for a in arms if a != "fp64_plain"]
    preds = {"linear": LinearPredictor(case.op), "euler": EulerPredictor(case.op),
             "midpoint": MidpointPredictor(case.op)}
    if net is not None:
        preds["learned"] = LearnedPredictor(case.op, net, norm)
        preds["learned_safeguarded"] = LearnedPredictor(case.op, net, norm, safeguard=True)
    # warm-up: workspaces of both inner precisions, library load, first launches
    for prec, cut in sorted({(ARMS[a][0], ARMS[a][2]) for a in arms}):
        run_arm(case, warmup_steps, prec, None, cut_off=cut)
    mass = lumped_mass_2d(case.nodes)
    u0 = case.op.to_host(case.u0)
    c0 = float(mass @ u0[0])
    out, ref, schedule, prev_prec = {}, None, None, None
    for a in arms:
        prec, kind, cut = ARMS[a]
        if kind is not None and kind not in preds:
            continue
        # the Newton workspace is rebuilt when the Krylov precision changes:
        # warm the new one up (GMRES graphs, first launches) outside the timing
        if prev_prec is not None and prec != prev_prec:
            run_arm(case, warmup_steps, prec, None, cut_off=cut)
        prev_prec = prec
        try:
            u, recs, wall = run_arm(case, n_steps, prec, preds.get(kind), schedule, cut_off=cut)
        except L.SintError as e:
            out[a] = {"failed": str(e)}
            continue
        if ref is None:
            ref, schedule = u, [r.dt for r in recs]
        out[a] = {
            "s_per_step": wall / len(recs),
            "wall_s": wall,
            "sim_time": float(sum(r.dt for r in recs)),
            "newton_iterations": int(sum(r.newton_iterations for r in recs)),
            "linear_iterations": int(sum(r.linear_iterations for r in recs)),
            "residual_evaluations": int(sum(r.residual_evaluations for r in recs)),
            "failed_tries": int(sum(r.failed_tries for r in recs)),
            # guess quality: |R(guess)| / |R(u_n)| over the predicted steps (geometric mean, worst)
            "guess_residual_ratio_gmean": _gmean([r.initial_residual / r.reference_residual for r in recs
                                                  if r.reference_residual > 0]),
            "guess_residual_ratio_max": max([r.initial_residual / r.reference_residual for r in recs
                                             if r.reference_residual > 0], default=None),
            "max_abs_diff_c": float(np.abs(u[0] - ref[0]).max()),
            "max_abs_diff_eta": float(np.abs(u[2:] - ref[2:]).max()),
            "int_c_rel_change": float(abs(mass @ u[0] - c0) / abs(c0)),
        }
    return out


def save_predictor(path, net: EquivariantNet, norm: Normaliser):
    """Trained parameters, architecture and normaliser as a NumPy .npz (no pickle)."""
    cfg = net.cfg
    np.savez(path, params=net.params.detach().cpu().numpy(), base=np.asarray(norm.base, np.float64),
             cfg=np.asarray([cfg.width, cfg.layers, cfg.grain_in, cfg.shared_in, cfg.shared_out, cfg.seed],
                            np.int64), slope=np.float64(cfg.slope), dim=np.int64(cfg.dim))


def load_predictor(path):
    """(net, normaliser) from save_predictor's file."""
    with np.load(path) as f:
        w, layers, gi, si, so, seed = (int(x) for x in f["cfg"])
        dim = int(f["dim"]) if "dim" in f.files else 2
        net = EquivariantNet(NetConfig(width=w, layers=layers, grain_in=gi, shared_in=si, shared_out=so,
                                       slope=float(f["slope"]), seed=seed, dim=dim))
        params = torch.as_tensor(f["params"], dtype=torch.float32)
        if params.numel() != net.n_params:
            raise ValueError(f"{path}: {params.numel()} parameters, the architecture needs {net.n_params}")
        net.load_params(params)
        return net, Normaliser([float(x) for x in f["base"]])


def train_learned_guess(train_seeds, n=512, n_circles=100, n_steps=200, net_cfg=None, train_cfg=None,
                        verbose=False, rmin=6.0, rmax=12.0):
    """FP64 trajectories over train_seeds, normaliser, Adam training.
    Returns (net, normaliser, trainer, info)."""
    t0 = time.perf_counter()
    trajs = [generate_trajectory(make_case(s, n, n_circles, rmin, rmax), n_steps) for s in train_seeds]
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    norm = fit_normaliser(trajs)
    net = EquivariantNet(net_cfg or NetConfig())
    tr = Trainer(net, norm, trajs, train_cfg)
    t_train = tr.train(verbose=verbose)
    info = {"trajectories": len(trajs), "triples": int(sum(t.n_triples() for t in trajs)),
            "grains": [t.case.G for t in trajs], "data_s": t_data, "train_s": t_train,
            "loss_history": tr.history, "params": net.n_params}
    return net, norm, tr, info
