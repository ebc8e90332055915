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
