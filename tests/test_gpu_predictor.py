"""CUDA kernels of the learned Newton guess against the NumPy reference
(oracle/predictor_ref.py, itself checked against finite differences).
FP32 kernels vs FP64 reference: relative tolerance 2e-5 of the tensor norm."""
import numpy as np
import pytest

from oracle import predictor_ref as R

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30)


def dev(x):
    return torch.tensor(np.asarray(x, np.float32), device="cuda").contiguous()


@pytest.mark.parametrize("N,Cin,Cout,H,W", [(2, 3, 5, 19, 23), (1, 32, 32, 33, 17), (3, 2, 1, 16, 16)])
def test_conv3x3_forward_and_gradients(N, Cin, Cout, H, W):
    from hpsint_b200 import predictor as P
    rng = np.random.default_rng(N * 100 + Cin)
    x, w, b = rng.normal(size=(N, Cin, H, W)), rng.normal(size=(Cout, Cin, 3, 3)), rng.normal(size=Cout)
    dout = rng.normal(size=(N, Cout, H, W))
    out = torch.empty((N, Cout, H, W), device="cuda")
    P.conv3x3(dev(x), dev(w), dev(b), out)
    assert rel(out.cpu().numpy(), R.conv3x3(x, w, b)) < 2e-5
    din = torch.empty((N, Cin, H, W), device="cuda")
    P.conv3x3_input_grad(dev(dout), dev(w), din)
    assert rel(din.cpu().numpy(), R.conv3x3_input_grad(dout, w)) < 2e-5
    dw, db = torch.zeros((Cout, Cin, 3, 3), device="cuda"), torch.zeros(Cout, device="cuda")
    P.conv3x3_weight_grad(dev(x), dev(dout), dw, db, P._Workspace(), accumulate=False)
    rw, rb = R.conv3x3_weight_grad(x, dout)
    assert rel(dw.cpu().numpy(), rw) < 2e-5 and rel(db.cpu().numpy(), rb) < 2e-5


def to_ref(net):
    return [{k: v.detach().double().cpu().numpy() for k, v in layer.items()} for layer in net.w]


def test_network_forward_backward_match_reference():
    from hpsint_b200 import predictor as P
    net = P.EquivariantNet(P.NetConfig(width=6, layers=3, seed=3))
    B, G, H, W = 2, 3, 18, 20
    rng = np.random.default_rng(5)
    xg, xs = rng.normal(size=(B * G, 2, H, W)), rng.normal(size=(B, 4, H, W))
    tg, ts = rng.normal(size=(B * G, 1, H, W)), rng.normal(size=(B, 2, H, W))
    yg, ys, cache = net.forward(dev(xg), dev(xs), B, G, keep=True)
    params = to_ref(net)
    ryg, rys, rcache = R.forward(params, xg, xs, B, G, net.cfg.slope)
    assert rel(yg.cpu().numpy(), ryg) < 2e-5 and rel(ys.cpu().numpy(), rys) < 2e-5
    net.zero_grad()
    net.backward(cache, dev(ryg - tg), dev(rys - ts), B, G)
    rgrads = R.backward(params, rcache, ryg - tg, rys - ts, B, G, net.cfg.slope)
    for l, layer in enumerate(net.g):
        for k, g in layer.items():
            assert rel(g.cpu().numpy(), rgrads[l][k]) < 1e-4, (l, k)


def test_network_is_grain_permutation_equivariant():
    from hpsint_b200 import predictor as P
    net = P.EquivariantNet(P.NetConfig(width=8, layers=3, seed=1))
    B, G, H, W = 1, 4, 16, 16
    rng = np.random.default_rng(2)
    xg, xs = rng.normal(size=(B * G, 2, H, W)), rng.normal(size=(B, 4, H, W))
    perm = [3, 1, 0, 2]
    yg, ys, _ = net.forward(dev(xg), dev(xs), B, G)
    yg2, ys2, _ = net.forward(dev(xg[perm]), dev(xs), B, G)
    assert torch.allclose(yg2, yg[perm], atol=1e-5) and torch.allclose(ys2, ys, atol=1e-5)


def test_adam_and_mse_match_reference():
    from hpsint_b200 import predictor as P
    net = P.EquivariantNet(P.NetConfig(width=4, layers=2))
    rng = np.random.default_rng(7)
    p0 = net.params.cpu().numpy().astype(np.float64)
    g = rng.normal(size=net.n_params)
    net.grads.copy_(dev(g))
    net.adam_step(lr=1e-2)
    net.adam_step(lr=1e-2)
    rp, rm, rv = R.adam(p0, g, np.zeros_like(p0), np.zeros_like(p0), 1e-2, 0.9, 0.999, 1e-8, 1)
    rp, rm, rv = R.adam(rp, g, rm, rv, 1e-2, 0.9, 0.999, 1e-8, 2)
    assert rel(net.params.cpu().numpy(), rp) < 1e-6
    pred, tgt, wt = rng.normal(size=1000), rng.normal(size=1000), rng.uniform(0, 1, 1000)
    grad = torch.empty(1000, device="cuda")
    loss = net.mse(dev(pred), dev(tgt), dev(wt), grad).item()
    assert abs(loss - np.sum(wt * (pred - tgt) ** 2) / 1000) < 1e-5 * loss
    assert rel(grad.cpu().numpy(), 2 * wt * (pred - tgt) / 1000) < 1e-6


@pytest.mark.parametrize("N,Cin,Cout,H,W", [(2, 32, 32, 33, 47), (1, 2, 32, 129, 129), (3, 4, 32, 16, 16),
                                            (1, 32, 32, 7, 300), (2, 32, 1, 40, 33), (1, 32, 2, 17, 65),
                                            (1, 5, 17, 21, 9)])
def test_tensor_core_conv_matches_fp32(N, Cin, Cout, H, W):
    """tcgen05 kind::tf32 convolution vs the FP32 kernel: TF32 operands keep
    10 mantissa bits, so the relative error of the output is ~1e-3 at most."""
    from hpsint_b200 import predictor as P
    rng = np.random.default_rng(Cin * 7 + H)
    x, w, b = rng.normal(size=(N, Cin, H, W)), rng.normal(size=(Cout, Cin, 3, 3)), rng.normal(size=Cout)
    ref = torch.empty((N, Cout, H, W), device="cuda")
    P.conv3x3(dev(x), dev(w), dev(b), ref)
    out = torch.full((N, Cout, H, W), 7.0, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    P.conv3x3_tc(dev(x), dev(w), dev(b), out, status)
    assert int(status.item()) == 0
    assert rel(out.cpu().numpy(), ref.cpu().numpy()) < 3e-3
    # accumulate mode adds onto the existing output
    P.conv3x3_tc(dev(x), dev(w), None, out, status, accumulate=True)
    P.conv3x3(dev(x), dev(w), None, ref, accumulate=True)
    assert rel(out.cpu().numpy(), ref.cpu().numpy()) < 3e-3


def test_network_inference_on_tensor_cores():
    from hpsint_b200 import predictor as P
    net = P.EquivariantNet(P.NetConfig(width=32, layers=4, seed=2))
    B, G, H, W = 1, 5, 40, 37
    rng = np.random.default_rng(9)
    xg, xs = dev(rng.normal(size=(B * G, 2, H, W))), dev(rng.normal(size=(B, 4, H, W)))
    yg, ys, _ = net.forward(xg, xs, B, G)
    yg2, ys2, _ = net.forward(xg, xs, B, G, tensor_cores=True)
    net.check_tensor_cores()
    assert rel(yg2.cpu().numpy(), yg.cpu().numpy()) < 1e-2 and rel(ys2.cpu().numpy(), ys.cpu().numpy()) < 1e-2


def test_tensor_core_conv_fused_epilogue():
    """act(conv + bias + out + addend[b // group]) against the FP32 kernel and torch arithmetic."""
    from hpsint_b200 import predictor as P
    rng = np.random.default_rng(4)
    Bg, grp, Cin, Cout, H, W = 6, 3, 32, 32, 19, 26
    x, w, b = rng.normal(size=(Bg, Cin, H, W)), rng.normal(size=(Cout, Cin, 3, 3)), rng.normal(size=Cout)
    q, o0 = rng.normal(size=(Bg // grp, Cout, H, W)), rng.normal(size=(Bg, Cout, H, W))
    ref = dev(o0)
    P.conv3x3(dev(x), dev(w), dev(b), ref, accumulate=True)
    ref = ref + dev(q).repeat_interleave(grp, dim=0)
    ref = torch.where(ref > 0, ref, 0.1 * ref)
    out = dev(o0)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    P.conv3x3_tc_ex(dev(x), dev(w), dev(b), out, status, accumulate=True, addend=dev(q), addend_group=grp, slope=0.1)
    assert int(status.item()) == 0
    assert rel(out.cpu().numpy(), ref.cpu().numpy()) < 3e-3


def test_curvature_loss_term_and_gradient_match_autograd():
    """lambda mean((Laplacian(w (p - t)))^2) and its gradient in p, against torch autograd."""
    import types
    from hpsint_b200 import learned_guess as LG
    from hpsint_b200 import predictor as P
    rng = np.random.default_rng(11)
    shape = (3, 2, 13, 17)
    p, t, w = dev(rng.normal(size=shape)), dev(rng.normal(size=shape)), dev(rng.uniform(0, 1, shape))
    grad = dev(rng.normal(size=shape))
    g0 = grad.clone()
    lam = 0.7
    me = types.SimpleNamespace(cfg=types.SimpleNamespace(smooth=lam), net=P.EquivariantNet(P.NetConfig(width=4, layers=2)),
                               _lap=torch.tensor([[0.0, 1, 0], [1, -4, 1], [0, 1, 0]], device="cuda").view(1, 1, 3, 3))
    loss = LG.Trainer._smooth_term(me, p, t, w, grad)
    pp = p.double().requires_grad_(True)
    e = (w.double() * (pp - t.double())).view(-1, 1, 13, 17)
    lap = torch.nn.functional.conv2d(e, me._lap.double(), padding=1)
    ref = lam * (lap ** 2).mean()
    ref.backward()
    assert abs(float(loss.item()) - float(ref.item())) <= 1e-5 * float(ref.item())
    assert rel((grad - g0).cpu().numpy(), pp.grad.cpu().numpy()) < 1e-5


# --- 3D: depth-padded windows [n][D + 2][C][H][W] -------------------------------------

def dev_padded(x):
    """[N][D][C][H][W] -> device [N][D + 2][C][H][W] with zero depth padding."""
    x = np.asarray(x, np.float32)
    out = np.zeros((x.shape[0], x.shape[1] + 2) + x.shape[2:], np.float32)
    out[:, 1:-1] = x
    return torch.tensor(out, device="cuda")


def inner(t):
    a = t.cpu().numpy()
    assert not a[:, 0].any() and not a[:, -1].any(), "depth padding must stay zero"
    return a[:, 1:-1]


@pytest.mark.parametrize("N,D,Cin,Cout,H,W", [(2, 5, 3, 4, 11, 13), (1, 3, 32, 32, 17, 9)])
def test_conv3x3x3_forward_and_gradients(N, D, Cin, Cout, H, W):
    from hpsint_b200 import predictor as P
    rng = np.random.default_rng(D * 10 + Cin)
    x, w3, b = rng.normal(size=(N, D, Cin, H, W)), rng.normal(size=(3, Cout, Cin, 3, 3)), rng.normal(size=Cout)
    dout = rng.normal(size=(N, D, Cout, H, W))
    out = torch.zeros((N, D + 2, Cout, H, W), device="cuda")
    P.conv3x3x3(dev_padded(x), dev(w3), dev(b), out)
    assert rel(inner(out), R.conv3x3x3(x, w3, b)) < 2e-5
    din = torch.zeros((N, D + 2, Cin, H, W), device="cuda")
    P.conv3x3x3_input_grad(dev_padded(dout), dev(w3), din)
    assert rel(inner(din), R.conv3x3x3_input_grad(dout, w3)) < 2e-5
    dw, db = torch.zeros((3, Cout, Cin, 3, 3), device="cuda"), torch.zeros(Cout, device="cuda")
    P.conv3x3x3_weight_grad(dev_padded(x), dev_padded(dout), dw, db, P._Workspace())
    rw, rb = R.conv3x3x3_weight_grad(x, dout)
    assert rel(dw.cpu().numpy(), rw) < 2e-5 and rel(db.cpu().numpy(), rb) < 2e-5
    # tensor cores (TF32 products)
    out_tc = torch.zeros_like(out)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    P.conv3x3x3(dev_padded(x), dev(w3), dev(b), out_tc, tc_status=status)
    assert int(status.item()) == 0
    assert rel(inner(out_tc), R.conv3x3x3(x, w3, b)) < 3e-3


def test_network3d_forward_backward_match_reference():
    from hpsint_b200 import predictor as P
    net = P.EquivariantNet(P.NetConfig(width=6, layers=3, seed=3, dim=3))
    B, G, D, H, W = 2, 3, 4, 9, 10
    rng = np.random.default_rng(6)
    xg, xs = rng.normal(size=(B * G, D, 2, H, W)), rng.normal(size=(B, D, 4, H, W))
    tg, ts = rng.normal(size=(B * G, D, 1, H, W)), rng.normal(size=(B, D, 2, H, W))
    yg, ys, cache = net.forward(dev_padded(xg), dev_padded(xs), B, G, keep=True)
    params = to_ref(net)
    ryg, rys, rcache = R.forward(params, xg, xs, B, G, net.cfg.slope)
    assert rel(inner(yg), ryg) < 2e-5 and rel(inner(ys), rys) < 2e-5
    net.zero_grad()
    net.backward(cache, dev_padded(ryg - tg), dev_padded(rys - ts), B, G)
    rgrads = R.backward(params, rcache, ryg - tg, rys - ts, B, G, net.cfg.slope)
    for l, layer in enumerate(net.g):
        for k, g in layer.items():
            assert rel(g.cpu().numpy(), rgrads[l][k]) < 1e-4, (l, k)
    # inference on the tensor cores (slice-shifted 3x3 convolutions)
    tyg, tys, _ = net.forward(dev_padded(xg), dev_padded(xs), B, G, tensor_cores=True, fused3d=False)
    net.check_tensor_cores()
    assert rel(inner(tyg), ryg) < 5e-3 and rel(inner(tys), rys) < 5e-3
    # one-pass FP32 inference (conv3d_fused): FP32 tolerance, zero padding written
    fyg, fys, _ = net.forward(dev_padded(xg), dev_padded(xs), B, G)
    assert rel(inner(fyg), ryg) < 2e-5 and rel(inner(fys), rys) < 2e-5


@pytest.mark.parametrize("S,D,c1,c2,cout,H,W,group", [(3, 5, 2, 0, 8, 11, 37, 3), (1, 11, 8, 8, 8, 9, 33, 1),
                                                        (2, 3, 4, 8, 2, 17, 13, 2), (2, 4, 8, 0, 1, 8, 32, 1),
                                                        (1, 9, 3, 5, 5, 10, 40, 1), (1, 6, 16, 16, 16, 12, 20, 1),
                                                        (1, 5, 32, 0, 32, 7, 35, 1)])
def test_conv3d_fused_matches_reference(S, D, c1, c2, cout, H, W, group):
    """The one-pass 3x3x3 convolution (two inputs, bias, addend broadcast over
    sample groups, leaky ReLU, accumulation) against the NumPy reference, over
    every output-channel instance (1, 2, 4, 8, 16, 32 and a padded 5), depths
    that are and are not multiples of the kernel's slice blocking, widths not
    a multiple of 32 and heights not a multiple of 8."""
    from hpsint_b200 import predictor as P
    rng = np.random.default_rng(S * 100 + D * 10 + cout)
    x1, w1 = rng.normal(size=(S, D, c1, H, W)), rng.normal(size=(3, cout, c1, 3, 3))
    b = rng.normal(size=cout)
    ref = R.conv3x3x3(x1, w1, b)
    x2 = w2 = None
    if c2:
        x2, w2 = rng.normal(size=(S, D, c2, H, W)), rng.normal(size=(3, cout, c2, 3, 3))
        ref = ref + R.conv3x3x3(x2, w2)
    add = rng.normal(size=(S // group, D, cout, H, W))
    ref = ref + np.repeat(add, group, axis=0)
    prev = rng.normal(size=(S, D, cout, H, W))
    out = dev_padded(prev)
    out[:, 0] = 7.0  # padding slices are overwritten with zero
    out[:, -1] = -3.0
    P.conv3d_fused(dev_padded(x1), dev(w1), out, x2=dev_padded(x2) if c2 else None, w2=dev(w2) if c2 else None,
                   bias=dev(b), addend=dev_padded(add), addend_group=group, slope=0.1, accumulate=True)
    expect = ref + prev
    expect = np.where(expect < 0, 0.1 * expect, expect)
    assert rel(inner(out), expect) < 2e-5
    # no bias, addend, activation or accumulation
    out2 = torch.full((S, D + 2, cout, H, W), 5.0, device="cuda")
    P.conv3d_fused(dev_padded(x1), dev(w1), out2)
    assert rel(inner(out2), R.conv3x3x3(x1, w1)) < 2e-5


def test_window3d_features_targets_and_guess():
    """sint_nn_features3d / targets3d / apply_guess3d against NumPy on a random
    3D state, with a window that reaches past the mesh (zeros there)."""
    import ctypes
    from hpsint_b200 import _lib as L
    nx, ny, nz, G = 7, 6, 5, 2
    N = nx * ny * nz
    ld = (N + 31) // 32 * 32
    rng = np.random.default_rng(11)
    u = [rng.normal(size=(2 + G, ld)) for _ in range(3)]  # u_{n-1}, u_n, u_{n+1}
    um, un, up = (torch.tensor(a, device="cuda") for a in u)
    scale = torch.tensor([1.5, 2.0, 0.5, 3.0, 1.25, 0.75], dtype=torch.float32, device="cuda")
    oscale = torch.tensor([2.0, 0.5, 4.0], dtype=torch.float32, device="cuda")
    x0, y0, z0, D, H, W, r = -1, 2, 1, 5, 5, 8, 0.8
    xg = torch.zeros((G, D + 2, 2, H, W), device="cuda")
    xs = torch.zeros((1, D + 2, 4, H, W), device="cuda")
    tg = torch.zeros((G, D + 2, 1, H, W), device="cuda")
    ts = torch.zeros((1, D + 2, 2, H, W), device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib = L.lib()
    L.check(lib.sint_nn_features3d_f64(p(un), p(um), ld, nx, ny, nz, G, x0, y0, z0, D, H, W, r, p(scale), p(xg),
                                       p(xs), 0, s), "features3d")
    L.check(lib.sint_nn_targets3d_f64(p(up), p(un), p(um), ld, nx, ny, nz, G, x0, y0, z0, D, H, W, r, p(oscale),
                                      p(tg), p(ts), 0, s), "targets3d")
    sc, osc = scale.cpu().numpy(), oscale.cpu().numpy()
    exg, exs = np.zeros((G, D, 2, H, W)), np.zeros((1, D, 4, H, W))
    etg, ets = np.zeros((G, D, 1, H, W)), np.zeros((1, D, 2, H, W))
    for z in range(D):
        for y in range(H):
            for x in range(W):
                zz, yy, xx = z0 + z, y0 + y, x0 + x
                if not (0 <= zz < nz and 0 <= yy < ny and 0 <= xx < nx):
                    continue
                n = (zz * ny + yy) * nx + xx
                for k in range(2 + G):
                    a, d = u[1][k, n], (u[1][k, n] - u[0][k, n]) * r
                    t = (u[2][k, n] - u[1][k, n]) - r * (u[1][k, n] - u[0][k, n])
                    if k < 2:
                        exs[0, z, 2 * k:2 * k + 2, y, x] = a * sc[2 * k], d * sc[2 * k + 1]
                        ets[0, z, k, y, x] = t * osc[k]
                    else:
                        exg[k - 2, z, :, y, x] = a * sc[4], d * sc[5]
                        etg[k - 2, z, 0, y, x] = t * osc[2]
    for got, ref in ((xg, exg), (xs, exs), (tg, etg), (ts, ets)):
        assert np.allclose(inner(got), ref, rtol=1e-6, atol=1e-6)
    # whole-plane window of mesh slices 1..4 with a halo of 1; guess for slices 2..3
    Dw, halo, zs, Dg = 4, 1, 2, 2
    yg = torch.tensor(rng.normal(size=(G, Dw + 2, 1, ny, nx)), dtype=torch.float32, device="cuda")
    ys = torch.tensor(rng.normal(size=(1, Dw + 2, 2, ny, nx)), dtype=torch.float32, device="cuda")
    guess = torch.zeros_like(un)
    L.check(lib.sint_nn_apply_guess3d_f64(p(un), p(um), ld, nx, ny, G, zs, Dg, halo, Dw, r, p(oscale), p(yg), p(ys),
                                          p(guess), s), "apply_guess3d")
    gy, sy, gs = yg.cpu().numpy(), ys.cpu().numpy(), guess.cpu().numpy()
    for z in range(zs, zs + Dg):
        wsl = 1 + halo + (z - zs)
        for k in range(2 + G):
            out = sy[0, wsl, k] if k < 2 else gy[k - 2, wsl, 0]
            sl = slice(z * nx * ny, (z + 1) * nx * ny)
            ref = u[1][k, sl] + r * (u[1][k, sl] - u[0][k, sl]) + out.ravel() / osc[min(k, 2)]
            assert np.allclose(gs[k, sl], ref, rtol=1e-6, atol=1e-6)
    assert not gs[:, :zs * nx * ny].any() and not gs[:, (zs + Dg) * nx * ny:N].any()
