"""Learned Newton initial guess: a grain-permutation-equivariant conv net.

The net predicts, for each node, the deviation of the next increment from
linear extrapolation,
    u_{n+1} - u_n - r (u_n - u_{n-1}),   r = dt_n / dt_{n-1},
from the last two states; the guess handed to Newton is
    u_n + r (u_n - u_{n-1}) + prediction.
It only replaces the initial iterate at the driver's predictor hook
(sintering/driver.h:2001-2058); the unchanged damped Newton solve to the same
tolerance decides the answer, so a bad prediction costs iterations, never
accuracy.

Equivariance: every order parameter eta_i is processed by the same weights
("grain streams"); grains interact only through the sum over grains (sum
pooling), and c, mu form a separate "shared stream".  Layer l maps
    grain:  h_i <- act(A * h_i + B * (sum_j h_j) + C * s + a)
    shared: s   <- act(D * s + E * (sum_j h_j) + d)
with 3x3 convolutions A..E (the last layer has no activation and outputs one
channel per grain and two shared channels: mu-free c and mu corrections).
Forward, backward and Adam run in the library's CUDA kernels (FP32); torch
only holds the device memory.
"""
import ctypes
import math
from dataclasses import dataclass

import torch

from . import _lib as L


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _s():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def conv3x3(x, w, bias, out, accumulate=False):
    """out (+)= conv(x, w) + bias; x [B][Cin][H][W], w [Cout][Cin][3][3]."""
    B, Cin, H, W = x.shape
    Cout = w.shape[0]
    L.check(L.lib().sint_nn_conv3x3_f32(_p(x), B, Cin, H, W, _p(w), _p(bias), _p(out), Cout, int(accumulate), _s()),
            "sint_nn_conv3x3_f32")


def conv3x3_tc(x, w, bias, out, status, accumulate=False):
    """conv3x3 on the tensor cores (TF32 products, FP32 accumulation); Cout <= 32, Cin <= 32.
    status: device int32 tensor, set to 1 by the kernel if a tensor-core wait timed out."""
    B, Cin, H, W = x.shape
    Cout = w.shape[0]
    L.check(L.lib().sint_nn_conv3x3_tc_f32(_p(x), B, Cin, H, W, _p(w), _p(bias), _p(out), Cout, int(accumulate),
                                           _p(status), _s()), "sint_nn_conv3x3_tc_f32")


def conv3x3_tc_ex(x, w, bias, out, status, accumulate=False, addend=None, addend_group=1, slope=None):
    """conv3x3_tc with the fused inference epilogue: out = act(conv + bias (+ out) (+ addend[b // group]))
    with act the leaky ReLU of `slope` (None: identity)."""
    B, Cin, H, W = x.shape
    Cout = w.shape[0]
    L.check(L.lib().sint_nn_conv3x3_tc_ex_f32(_p(x), B, Cin, H, W, _p(w), _p(bias), _p(out), Cout, int(accumulate),
                                              _p(addend), int(addend_group), int(slope is not None),
                                              float(slope or 0.0), _p(status), _s()), "sint_nn_conv3x3_tc_ex_f32")


def conv3x3_input_grad(dout, w, din, accumulate=False, wT=None):
    """din (+)= d(conv(x, w))/dx applied to dout (convolution with the flipped kernel)."""
    Cout, Cin = w.shape[0], w.shape[1]
    if wT is None:
        wT = torch.empty((Cin, Cout, 3, 3), dtype=torch.float32, device="cuda")
    L.check(L.lib().sint_nn_conv3x3_flip_f32(_p(w), Cout, Cin, _p(wT), _s()), "sint_nn_conv3x3_flip_f32")
    conv3x3(dout, wT, None, din, accumulate)


class _Workspace:
    """Grow-only scratch for the weight-gradient and loss reductions."""

    def __init__(self):
        self.buf = torch.empty(0, dtype=torch.float32, device="cuda")
        self.dbuf = torch.empty(L.lib().sint_nn_mse_workspace(), dtype=torch.float64, device="cuda")

    def get(self, n):
        if self.buf.numel() < n:
            self.buf = torch.empty(int(n * 1.25) + 1024, dtype=torch.float32, device="cuda")
        return self.buf


def conv3x3_weight_grad(x, dout, dw, db, ws, accumulate=True):
    B, Cin, H, W = x.shape
    Cout = dout.shape[1]
    n = L.lib().sint_nn_conv3x3_wgrad_workspace(B, Cin, Cout, H, W)
    work = ws.get(n)
    L.check(L.lib().sint_nn_conv3x3_wgrad_f32(_p(x), _p(dout), B, Cin, Cout, H, W, _p(dw), _p(db), int(accumulate),
                                              _p(work), _s()), "sint_nn_conv3x3_wgrad_f32")


# --- 3D: depth-padded windows [sample][D + 2][channels][H][W] ----------------------
# Every depth slice of every sample is one contiguous [C][H][W] image; a 3x3x3
# convolution is three 3x3 convolutions of the slice batch shifted by -1, 0,
# +1 slices (weights w3 [3][Cout][Cin][3][3], index 0 = the slice below), the
# zero slices around each sample being the depth padding.  Shifted batches
# also write the padding slices of the output (across sample boundaries);
# they are zeroed after every convolution.

def _slices(t):
    S, D2, C, H, W = t.shape
    return t.view(S * D2, C, H, W)


def zero_pads(t):
    L.check(L.lib().sint_nn_zero_pad_slices_f32(_p(t), t.shape[0], t.shape[1], t[0, 0].numel(), _s()),
            "sint_nn_zero_pad_slices_f32")


def conv3x3x3(x, w3, bias, out, accumulate=False, tc_status=None):
    """out (+)= conv(x, w3) + bias on depth-padded windows; tc_status: run on the
    tensor cores (TF32 products) and report timed-out waits there."""
    xs, os_ = _slices(x), _slices(out)
    n = xs.shape[0]
    for j, dz in enumerate((-1, 0, 1)):
        src, dst = xs[1 + dz:n - 1 + dz], os_[1:n - 1]
        acc, b = accumulate or j > 0, (bias if j == 0 else None)
        if tc_status is not None:
            conv3x3_tc(src, w3[j], b, dst, tc_status, acc)
        else:
            conv3x3(src, w3[j], b, dst, acc)
    zero_pads(out)


def conv3d_fused(x1, w1, out, x2=None, w2=None, bias=None, addend=None, addend_group=1, slope=None,
                 accumulate=False):
    """Inference form of the 3x3x3 convolution on depth-padded windows, one
    pass: out = act(conv(x1, w1) (+ conv(x2, w2)) + bias (+ addend broadcast
    over groups of addend_group samples) (+ out)), act = leaky ReLU with
    `slope` (None: identity); the output's padding slices are written as zero."""
    S, D2, c1, H, W = x1.shape
    c2 = x2.shape[2] if x2 is not None else 0
    L.check(L.lib().sint_nn_conv3d_f32(S, D2 - 2, H, W, _p(x1), c1, _p(w1), _p(x2), c2, _p(w2), _p(bias), _p(addend),
                                       addend_group, 1 if slope is not None else 0,
                                       float(slope) if slope is not None else 0.0, _p(out), out.shape[2],
                                       int(accumulate), _s()), "sint_nn_conv3d_f32")


def conv3x3x3_input_grad(dout, w3, din, accumulate=False):
    """din (+)= d(conv(x, w3))/dx applied to dout: din[z] = sum_dz W_dz^T * dout[z - dz]."""
    ds, dis = _slices(dout), _slices(din)
    n = ds.shape[0]
    for j, dz in enumerate((-1, 0, 1)):
        conv3x3_input_grad(ds[1 - dz:n - 1 - dz], w3[j], dis[1:n - 1], accumulate or j > 0)
    zero_pads(din)


def conv3x3x3_weight_grad(x, dout, dw3, db, ws):
    """dw3[dz] += sum over slices of x[z + dz] correlated with dout[z]; db += sum of dout."""
    xs, ds = _slices(x), _slices(dout)
    n = xs.shape[0]
    for j, dz in enumerate((-1, 0, 1)):
        conv3x3_weight_grad(xs[1 + dz:n - 1 + dz], ds[1:n - 1], dw3[j], db if j == 1 else None, ws)


def leaky(x, y, slope):
    L.check(L.lib().sint_nn_leaky_relu_f32(x.numel(), slope, _p(x), _p(y), _s()), "sint_nn_leaky_relu_f32")


def leaky_bwd(pre, dy, dx, slope):
    L.check(L.lib().sint_nn_leaky_relu_bwd_f32(pre.numel(), slope, _p(pre), _p(dy), _p(dx), _s()),
            "sint_nn_leaky_relu_bwd_f32")


def grain_sum(h, B, G, P):
    chw = h[0].numel()
    L.check(L.lib().sint_nn_grain_sum_f32(_p(h), B, G, chw, _p(P), _s()), "sint_nn_grain_sum_f32")


def grain_bcast_add(Q, B, G, Z):
    chw = Q[0].numel()
    L.check(L.lib().sint_nn_grain_bcast_add_f32(_p(Q), B, G, chw, _p(Z), _s()), "sint_nn_grain_bcast_add_f32")


@dataclass
class NetConfig:
    width: int = 32
    layers: int = 4
    dim: int = 2          # 3: 3x3x3 convolutions on depth-padded windows
    grain_in: int = 2     # eta_i, extrapolated eta_i increment
    shared_in: int = 4    # c, c increment, mu, mu increment
    shared_out: int = 2   # corrections of c and mu (one grain channel per eta_i)
    slope: float = 0.1    # leaky-ReLU slope
    seed: int = 0


class EquivariantNet:
    """Parameters live in one flat FP32 device tensor (views per weight); so do
    their gradients and the Adam moments."""

    NAMES = ("A", "B", "C", "D", "E", "a", "d")

    def __init__(self, cfg: NetConfig = None):
        self.cfg = cfg = cfg or NetConfig()
        self.dims = []
        cg, cs = cfg.grain_in, cfg.shared_in
        for l in range(cfg.layers):
            last = l == cfg.layers - 1
            go, so = (1, cfg.shared_out) if last else (cfg.width, cfg.width)
            self.dims.append((cg, cs, go, so))
            cg, cs = go, so
        self.shapes = []
        cw = (lambda co, ci: (co, ci, 3, 3)) if cfg.dim == 2 else (lambda co, ci: (3, co, ci, 3, 3))
        for (cg, cs, go, so) in self.dims:
            self.shapes.append({"A": cw(go, cg), "B": cw(go, cg), "C": cw(go, cs), "D": cw(so, cs),
                                "E": cw(so, cg), "a": (go,), "d": (so,)})
        self.taps = 9 if cfg.dim == 2 else 27
        n = sum(math.prod(s) for sh in self.shapes for s in sh.values())
        self.n_params = n
        self.params = torch.zeros(n, dtype=torch.float32, device="cuda")
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_count = 0
        self.w = self._views(self.params)
        self.g = self._views(self.grads)
        self.ws = _Workspace()
        self.tc_status = torch.zeros(1, dtype=torch.int32, device="cuda")
        self._init(cfg.seed)

    def _views(self, flat):
        out, off = [], 0
        for sh in self.shapes:
            d = {}
            for k in self.NAMES:
                s = sh[k]
                d[k] = flat[off:off + math.prod(s)].view(s)
                off += math.prod(s)
            out.append(d)
        return out

    def _init(self, seed):
        """He-normal weights for the hidden layers, small output layer, zero biases."""
        gen = torch.Generator().manual_seed(seed)
        for l, (cg, cs, go, so) in enumerate(self.dims):
            last = l == len(self.dims) - 1
            for k in ("A", "B", "C"):
                fan = self.taps * (2 * cg + cs)
                std = math.sqrt(2.0 / fan) * (0.1 if last else 1.0)
                self.w[l][k].copy_(torch.randn(self.shapes[l][k], generator=gen) * std)
            for k in ("D", "E"):
                fan = self.taps * (cs + cg)
                std = math.sqrt(2.0 / fan) * (0.1 if last else 1.0)
                self.w[l][k].copy_(torch.randn(self.shapes[l][k], generator=gen) * std)

    # -- forward -------------------------------------------------------------
    def forward(self, xg, xs, B, G, keep=False, tensor_cores=False, fused3d=True, ws=None):
        """xg [B*G][grain_in][H][W], xs [B][shared_in][H][W] -> (yg [B*G][1], ys [B][2]).
        tensor_cores: run the convolutions on the tensor cores (TF32 products,
        FP32 accumulation; inference) instead of the FP32 kernel.
        3D inference (keep False) with fused3d: one-pass FP32 3x3x3
        convolutions with the layer's sums, bias and activation fused
        (conv3d_fused; tensor_cores does not apply); ws: a dict that keeps
        the activation buffers of that path between calls (the caller owns
        it and must not run two calls with one ws at the same time)."""
        H, W = xs.shape[-2], xs.shape[-1]
        if self.cfg.dim == 2 and tensor_cores and not keep and max(max(d) for d in self.dims) <= 32:
            return self._forward_fused(xg, xs, B, G, H, W)
        if self.cfg.dim == 3 and fused3d and not keep and max(max(d) for d in self.dims) <= 32:
            return self._forward_fused3d(xg, xs, B, G, H, W, ws)
        cache = []
        hg, hs = xg, xs
        # 2D: [n][C][H][W]; 3D: [n][D + 2][C][H][W]
        shape = (lambda n, c: (n, c, H, W)) if self.cfg.dim == 2 else (lambda n, c: (n, xs.shape[1], c, H, W))

        def conv(x, wt, bias, out, accumulate=False):
            tc = tensor_cores and wt.shape[-4] <= 32 and wt.shape[-3] <= 32
            if self.cfg.dim == 3:
                conv3x3x3(x, wt, bias, out, accumulate, self.tc_status if tc else None)
            elif tc:
                conv3x3_tc(x, wt, bias, out, self.tc_status, accumulate)
            else:
                conv3x3(x, wt, bias, out, accumulate)

        for l, (cg, cs, go, so) in enumerate(self.dims):
            w = self.w[l]
            P = torch.empty(shape(B, cg), dtype=torch.float32, device="cuda")
            grain_sum(hg, B, G, P)
            Zg = torch.empty(shape(B * G, go), dtype=torch.float32, device="cuda")
            conv(hg, w["A"], w["a"], Zg)
            Q = torch.empty(shape(B, go), dtype=torch.float32, device="cuda")
            conv(P, w["B"], None, Q)
            conv(hs, w["C"], None, Q, accumulate=True)
            grain_bcast_add(Q, B, G, Zg)
            Zs = torch.empty(shape(B, so), dtype=torch.float32, device="cuda")
            conv(hs, w["D"], w["d"], Zs)
            conv(P, w["E"], None, Zs, accumulate=True)
            if keep:
                cache.append((hg, hs, P, Zg, Zs))
            if l < len(self.dims) - 1:
                ng, ns = torch.empty_like(Zg), torch.empty_like(Zs)
                leaky(Zg, ng, self.cfg.slope)
                leaky(Zs, ns, self.cfg.slope)
                hg, hs = ng, ns
            else:
                hg, hs = Zg, Zs
        return hg, hs, cache

    def _forward_fused(self, xg, xs, B, G, H, W):
        """Inference on the tensor cores with fused epilogues: per layer
        P = sum_i h_i;  Q = B*P + C*s;  h_i <- act(A*h_i + a + Q)  (one conv);
        s <- act(D*s + d + E*P)  (the activation in the second conv)."""
        hg, hs = xg, xs
        n = len(self.dims)
        st = self.tc_status
        for l, (cg, cs, go, so) in enumerate(self.dims):
            w = self.w[l]
            slope = self.cfg.slope if l < n - 1 else None
            P = torch.empty((B, cg, H, W), dtype=torch.float32, device="cuda")
            grain_sum(hg, B, G, P)
            Q = torch.empty((B, go, H, W), dtype=torch.float32, device="cuda")
            conv3x3_tc(P, w["B"], None, Q, st)
            conv3x3_tc(hs, w["C"], None, Q, st, accumulate=True)
            Zg = torch.empty((B * G, go, H, W), dtype=torch.float32, device="cuda")
            conv3x3_tc_ex(hg, w["A"], w["a"], Zg, st, addend=Q, addend_group=G, slope=slope)
            Zs = torch.empty((B, so, H, W), dtype=torch.float32, device="cuda")
            conv3x3_tc(hs, w["D"], w["d"], Zs, st)
            conv3x3_tc_ex(P, w["E"], None, Zs, st, accumulate=True, slope=slope)
            hg, hs = Zg, Zs
        return hg, hs, []

    def _forward_fused3d(self, xg, xs, B, G, H, W, ws=None):
        """3D inference, three one-pass convolutions per layer:
        P = sum_i h_i;  Q = B*P + C*s;  h_i <- act(A*h_i + a + Q);
        s <- act(D*s + d + E*P).  Buffers per layer and role, kept in ws."""
        def buf(key, shape):
            t = ws.get(key) if ws is not None else None
            if t is None or tuple(t.shape) != shape:
                t = torch.empty(shape, dtype=torch.float32, device="cuda")
                if ws is not None:
                    ws[key] = t
            return t

        hg, hs = xg, xs
        n, D2 = len(self.dims), xs.shape[1]
        for l, (cg, cs, go, so) in enumerate(self.dims):
            w = self.w[l]
            slope = self.cfg.slope if l < n - 1 else None
            P = buf(("P", l), (B, D2, cg, H, W))
            grain_sum(hg, B, G, P)
            Q = buf(("Q", l), (B, D2, go, H, W))
            conv3d_fused(P, w["B"], Q, x2=hs, w2=w["C"])
            Zg = buf(("Zg", l), (B * G, D2, go, H, W))
            conv3d_fused(hg, w["A"], Zg, bias=w["a"], addend=Q, addend_group=G, slope=slope)
            Zs = buf(("Zs", l), (B, D2, so, H, W))
            conv3d_fused(hs, w["D"], Zs, x2=P, w2=w["E"], bias=w["d"], slope=slope)
            hg, hs = Zg, Zs
        return hg, hs, []

    # -- backward ------------------------------------------------------------
    def backward(self, cache, dyg, dys, B, G):
        """Accumulate parameter gradients of a loss with output gradients (dyg, dys)."""
        dZg, dZs = dyg, dys
        for l in reversed(range(len(self.dims))):
            hg, hs, P, Zg, Zs = cache[l]
            if l < len(self.dims) - 1:
                leaky_bwd(Zg, dZg, dZg, self.cfg.slope)
                leaky_bwd(Zs, dZs, dZs, self.cfg.slope)
            w, g = self.w[l], self.g[l]
            cg, cs, go, so = self.dims[l]
            H, W = hs.shape[-2], hs.shape[-1]
            if self.cfg.dim == 2:
                shape = lambda n, c: (n, c, H, W)
                wgrad, igrad = conv3x3_weight_grad, conv3x3_input_grad
            else:
                shape = lambda n, c: (n, hs.shape[1], c, H, W)
                wgrad, igrad = conv3x3x3_weight_grad, conv3x3x3_input_grad
            dQ = torch.empty(shape(B, go), dtype=torch.float32, device="cuda")
            grain_sum(dZg, B, G, dQ)
            wgrad(hg, dZg, g["A"], g["a"], self.ws)
            wgrad(P, dQ, g["B"], None, self.ws)
            wgrad(hs, dQ, g["C"], None, self.ws)
            wgrad(hs, dZs, g["D"], g["d"], self.ws)
            wgrad(P, dZs, g["E"], None, self.ws)
            if l == 0:
                break
            dhg = torch.empty(shape(B * G, cg), dtype=torch.float32, device="cuda")
            igrad(dZg, w["A"], dhg)
            dP = torch.empty(shape(B, cg), dtype=torch.float32, device="cuda")
            igrad(dQ, w["B"], dP)
            igrad(dZs, w["E"], dP, accumulate=True)
            grain_bcast_add(dP, B, G, dhg)
            dhs = torch.empty(shape(B, cs), dtype=torch.float32, device="cuda")
            igrad(dQ, w["C"], dhs)
            igrad(dZs, w["D"], dhs, accumulate=True)
            dZg, dZs = dhg, dhs

    def check_tensor_cores(self):
        """Raise if a tensor-core convolution reported a timed-out wait (synchronises)."""
        if int(self.tc_status.item()) != 0:
            self.tc_status.zero_()
            raise L.SintError(3, "EquivariantNet",
                              "tensor-core convolution timed out waiting for its MMAs")

    def zero_grad(self):
        self.grads.zero_()

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        L.check(L.lib().sint_nn_adam_f32(self.n_params, _p(self.params), _p(self.grads), _p(self.m), _p(self.v),
                                         lr, beta1, beta2, eps, self.step_count, _s()), "sint_nn_adam_f32")

    def mse(self, pred, target, weight, grad):
        """loss (device double) and, into grad, its gradient (mean over elements)."""
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        L.check(L.lib().sint_nn_mse_f32(pred.numel(), _p(pred), _p(target), _p(weight), _p(grad), _p(loss),
                                        _p(self.ws.dbuf), _s()), "sint_nn_mse_f32")
        return loss

    def state_dict(self):
        return {"cfg": self.cfg.__dict__, "params": self.params.detach().cpu()}

    def load_params(self, flat):
        self.params.copy_(flat.to(self.params.device))
