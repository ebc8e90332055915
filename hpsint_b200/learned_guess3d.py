"""Learned Newton initial guess in 3D: data, training and the predictor.

The 3D counterpart of learned_guess (same network family, same targets and
normalisation): the grain-permutation-equivariant net with 3x3x3
convolutions (predictor.NetConfig(dim=3)), trained on random cubic windows
of FP64 trajectories of small 3D packings (lognormal spheres, tensorial
mobility, as the 256^3 packing solve uses), and applied to a whole mesh in
slabs of depth slices so that the activations of a large mesh fit in HBM.

Windows are depth-padded tensors [sample][D + 2][channels][H][W] (one zero
slice before and after every sample; sint_nn_features3d_f64).  Nothing here
decides the answer: each step is still the damped Newton-Krylov solve to the
same tolerance (sintering/driver.h:2001-2058 is the predictor hook).
"""
import math
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from . import packings as PK
from . import predictor as NP
from .learned_guess import (IncrementScales, LinearPredictor, Normaliser, Trainer, TrainConfig, _p, _s,
                            _triple_scales, fit_normaliser, generate_trajectory, model_params)
from .operator import Mesh, SinteringOperatorGeneric
from .predictor import EquivariantNet, NetConfig


@dataclass
class Case3D:
    """One 3D packing: its operator and initial state (device)."""
    seed: int
    n: int
    G: int
    op: SinteringOperatorGeneric
    u0: torch.Tensor

    @property
    def nodes(self):
        return self.n + 1


def make_case3d(seed, n=64, n_spheres=12, median=8.0, sigma=0.25, max_grains=8, tensorial=True):
    """Lognormal sphere packing on [0, n]^3 (packings.lognormal_packing_3d),
    width-2 tanh profiles, hpsint's default constants."""
    centers, radii, colours = PK.lognormal_packing_3d(n=n, n_spheres=n_spheres, median=median, sigma=sigma,
                                                      max_grains=max_grains, seed=seed)
    G = int(colours.max()) + 1
    u0 = PK.initial_state(3, (n, n, n), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), centers, radii, colours, width=2.0)
    op = SinteringOperatorGeneric(Mesh(3, (n, n, n)), model_params(G, tensorial))
    return Case3D(seed, n, G, op, op.to_device(u0))


class WindowSampler3D:
    """Random cubic windows of random triples, drawn where the window holds
    material (max c > 0.01 over a stride-8 grid of origins) and reaching up to
    `margin` nodes past the mesh, where the features read zero."""

    def __init__(self, trajs, window, margin, rng):
        self.trajs = [t for t in trajs if t.n_triples() > 0]
        if not self.trajs:
            raise ValueError("no trajectory with at least one (u_{n-1}, u_n, u_{n+1}) triple")
        self.window, self.margin, self.rng = window, margin, rng
        self.origins = []
        for tr in self.trajs:
            nn = tr.case.nodes
            c = tr.states[0][0, :tr.case.op.N].view(nn, nn, nn).cpu().numpy()  # [z][y][x]
            lo, hi = -margin, nn - window + margin
            cand = []
            for z0 in range(lo, max(lo, hi) + 1, 8):
                for y0 in range(lo, max(lo, hi) + 1, 8):
                    for x0 in range(lo, max(lo, hi) + 1, 8):
                        zs, ys, xs = max(0, z0), max(0, y0), max(0, x0)
                        if c[zs:z0 + window, ys:y0 + window, xs:x0 + window].max(initial=0.0) > 0.01:
                            cand.append((x0, y0, z0))
            self.origins.append(cand or [(lo, lo, lo)])

    def draw(self):
        ti = int(self.rng.integers(len(self.trajs)))
        tr, cand = self.trajs[ti], self.origins[ti]
        hi = tr.case.nodes - self.window + self.margin
        out = []
        for _ in range(self.batch_size):
            k = int(self.rng.integers(1, len(tr.states) - 1))
            o = cand[int(self.rng.integers(len(cand)))]
            j = self.rng.integers(-4, 5, size=3)
            x0, y0, z0 = (int(min(max(o[d] + j[d], -self.margin), hi)) for d in range(3))
            out.append((k, x0, y0, z0))
        return tr, out


class Trainer3D(Trainer):
    """Trainer on cubic windows: border-masked MSE plus the curvature term
    with the 7-point Laplacian (a 3x3x3 kernel applied by the library's
    convolution)."""

    def __init__(self, net: EquivariantNet, norm: Normaliser, trajs, cfg: TrainConfig = None):
        if net.cfg.dim != 3:
            raise ValueError("Trainer3D needs a NetConfig(dim=3) network")
        self.net, self.norm, self.cfg = net, norm, cfg or TrainConfig(window=24, batch=2)
        self.rng = np.random.default_rng(self.cfg.seed)
        self.margin = net.cfg.layers
        self.sampler = WindowSampler3D(trajs, self.cfg.window, self.margin, self.rng)
        self.sampler.batch_size = self.cfg.batch
        base, inc = norm.device(), IncrementScales()
        self.scales = {id(tr): _triple_scales(tr, base, inc) for tr in self.sampler.trajs}
        self.history = []
        self._bufs = {}
        lap = torch.zeros((3, 1, 1, 3, 3), dtype=torch.float32, device="cuda")
        lap[1, 0, 0] = torch.tensor([[0.0, 1.0, 0.0], [1.0, -6.0, 1.0], [0.0, 1.0, 0.0]])
        lap[0, 0, 0, 1, 1] = lap[2, 0, 0, 1, 1] = 1.0
        self._lap3 = lap

    def _buffers(self, G):
        if G not in self._bufs:
            B, Wn = self.cfg.batch, self.cfg.window
            f = lambda n, c: torch.zeros((n, Wn + 2, c, Wn, Wn), dtype=torch.float32, device="cuda")
            self._bufs[G] = dict(xg=f(B * G, 2), xs=f(B, 4), tg=f(B * G, 1), ts=f(B, 2), wg=f(B * G, 1),
                                 ws=f(B, 2), dyg=f(B * G, 1), dys=f(B, 2))
        return self._bufs[G]

    def _window_mask(self, x0, y0, z0, nodes):
        Wn, m = self.cfg.window, self.margin
        mask = torch.zeros((Wn, Wn, Wn), dtype=torch.float32, device="cuda")
        lo = [max(m, -o) for o in (z0, y0, x0)]
        hi = [min(Wn - m, nodes - o) for o in (z0, y0, x0)]
        if all(a < b for a, b in zip(lo, hi)):
            mask[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = 1.0
        return mask

    def fill_batch(self):
        tr, picks = self.sampler.draw()
        G, nodes, ld = tr.case.G, tr.case.nodes, tr.case.op.ld
        b = self._buffers(G)
        Wn = self.cfg.window
        lib = L.lib()
        sc, osc = self.scales[id(tr)]
        for i, (k, x0, y0, z0) in enumerate(picks):
            un, um, up = tr.states[k], tr.states[k - 1], tr.states[k + 1]
            r = tr.dts[k] / tr.dts[k - 1]
            L.check(lib.sint_nn_features3d_f64(_p(un), _p(um), ld, nodes, nodes, nodes, G, x0, y0, z0, Wn, Wn, Wn, r,
                                               _p(sc[k]), _p(b["xg"]), _p(b["xs"]), i, _s()),
                    "sint_nn_features3d_f64")
            L.check(lib.sint_nn_targets3d_f64(_p(up), _p(un), _p(um), ld, nodes, nodes, nodes, G, x0, y0, z0, Wn, Wn,
                                              Wn, r, _p(osc[k]), _p(b["tg"]), _p(b["ts"]), i, _s()),
                    "sint_nn_targets3d_f64")
            mask = self._window_mask(x0, y0, z0, nodes)  # [z][y][x]
            b["wg"][i * G:(i + 1) * G, 1:-1, 0].copy_(mask.expand(G, Wn, Wn, Wn))
            b["ws"][i, 1:-1].copy_(mask.unsqueeze(1).expand(Wn, 2, Wn, Wn))
        return G, b

    def _smooth_term(self, pred, target, weight, grad):
        """lambda mean((Delta (w (pred - target)))^2) with the 7-point Laplacian
        (symmetric, so its transpose is itself); adds lambda 2/n w
        Delta(Delta(w e)) to grad (grad may be None)."""
        lam = self.cfg.smooth
        S, D2, C, H, W = pred.shape
        e = torch.empty_like(pred)
        L.check(L.lib().sint_nn_weighted_diff_f32(pred.numel(), _p(pred), _p(target), _p(weight), _p(e), _s()),
                "sint_nn_weighted_diff_f32")
        # channels as samples: [S][D2][C][H][W] -> per channel a 1-channel window
        ec = e.permute(0, 2, 1, 3, 4).contiguous().view(S * C, D2, 1, H, W)
        lap = torch.zeros_like(ec)
        NP.conv3x3x3(ec, self._lap3, None, lap)
        g_l = torch.zeros_like(ec) if grad is not None else None
        loss = self.net.mse(lap, torch.zeros_like(lap), None, g_l)
        if grad is not None:
            q = torch.zeros_like(ec)
            NP.conv3x3x3(g_l, self._lap3, None, q)
            qb = q.view(S, C, D2, H, W).permute(0, 2, 1, 3, 4).contiguous()
            L.check(L.lib().sint_nn_mul_add_f32(pred.numel(), lam, _p(weight), _p(qb), _p(grad), _s()),
                    "sint_nn_mul_add_f32")
        return loss * lam


class LearnedPredictor3D:
    """Whole-mesh inference in slabs of `slab` depth slices (each with a halo
    of `layers` slices, the network's receptive field in depth):
    features -> net -> guess u_n + r (u_n - u_{n-1}) + output / oscale.  FP32
    network (one-pass FP32 3x3x3 convolutions with the layer's sums and
    activations fused; fused=False: slice-shifted 3x3 convolutions, on the
    tensor cores with tensor_cores), FP64 guess.  safeguard: keep the smaller
    residual of this guess and hpsint's linear one (device only)."""

    def __init__(self, op: SinteringOperatorGeneric, net: EquivariantNet, norm: Normaliser, slab=64,
                 tensor_cores=True, safeguard=False, fused=True):
        if op.mesh.dim != 3 or net.cfg.dim != 3:
            raise ValueError("LearnedPredictor3D needs a 3D mesh and a NetConfig(dim=3) network")
        self.op, self.net, self.tensor_cores, self.safeguard = op, net, tensor_cores, safeguard
        self.fused = fused
        self.ws = {}  # activation buffers of the fused network, kept between calls
        self.base, self.inc = norm.device(), IncrementScales()
        self.scale = torch.ones(6, dtype=torch.float32, device="cuda")
        self.oscale = torch.ones(3, dtype=torch.float32, device="cuda")
        self.nx, self.ny, self.nz = (op.mesh.n_cells[d] + 1 for d in range(3))
        self.halo = net.cfg.layers
        # slabs of at most `slab` slices, split evenly (no short last slab
        # computed over a full window)
        n_slabs = -(-self.nz // max(1, slab))
        self.slab = -(-self.nz // n_slabs)
        G = op.params.n_grains
        Dw = self.slab + 2 * self.halo
        f = lambda n, c: torch.zeros((n, Dw + 2, c, self.ny, self.nx), dtype=torch.float32, device="cuda")
        self.xg, self.xs = f(G, 2), f(1, 4)
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
        h, Dw = self.halo, self.slab + 2 * self.halo
        for z0 in range(0, self.nz, self.slab):
            D = min(self.slab, self.nz - z0)
            # window of mesh slices z0 - h .. z0 - h + Dw - 1 (zeros beyond the mesh)
            L.check(lib.sint_nn_features3d_f64(_p(history[0]), _p(history[1]), op.ld, self.nx, self.ny, self.nz, G,
                                               0, 0, z0 - h, Dw, self.ny, self.nx, r, _p(self.scale), _p(self.xg),
                                               _p(self.xs), 0, _s()), "sint_nn_features3d_f64")
            yg, ys, _ = self.net.forward(self.xg, self.xs, 1, G, tensor_cores=self.tensor_cores, fused3d=self.fused,
                                         ws=self.ws)
            L.check(lib.sint_nn_apply_guess3d_f64(_p(history[0]), _p(history[1]), op.ld, self.nx, self.ny, G, z0, D,
                                                  h, Dw, r, _p(self.oscale), _p(yg), _p(ys), _p(self.guess), _s()),
                    "sint_nn_apply_guess3d_f64")
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


def train_learned_guess3d(train_seeds, n=64, n_spheres=12, n_steps=60, net_cfg=None, train_cfg=None,
                          verbose=False, median=8.0, sigma=0.25, max_grains=8):
    """FP64 trajectories of 3D packings over train_seeds, normaliser, Adam.
    Returns (net, normaliser, trainer, info)."""
    t0 = time.perf_counter()
    trajs = [generate_trajectory(make_case3d(s, n, n_spheres, median, sigma, max_grains), n_steps)
             for s in train_seeds]
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    norm = fit_normaliser(trajs)
    net = EquivariantNet(net_cfg or NetConfig(dim=3, width=16, layers=3))
    tr = Trainer3D(net, norm, trajs, train_cfg)
    t_train = tr.train(verbose=verbose)
    info = {"trajectories": len(trajs), "triples": int(sum(t.n_triples() for t in trajs)),
            "grains": [t.case.G for t in trajs], "data_s": t_data, "train_s": t_train,
            "loss_history": tr.history, "params": net.n_params,
            "steps": [len(t.states) - 1 for t in trajs]}
    return net, norm, tr, info
