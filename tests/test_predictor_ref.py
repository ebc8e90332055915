"""The NumPy reference of the learned-guess network against finite differences
and its own symmetry (CPU only)."""
import numpy as np

from oracle import predictor_ref as R


def small_net(rng, dims):
    params = []
    for (cg, cs, go, so) in dims:
        params.append({"A": rng.normal(0, .3, (go, cg, 3, 3)), "B": rng.normal(0, .3, (go, cg, 3, 3)),
                       "C": rng.normal(0, .3, (go, cs, 3, 3)), "D": rng.normal(0, .3, (so, cs, 3, 3)),
                       "E": rng.normal(0, .3, (so, cg, 3, 3)), "a": rng.normal(0, .1, go),
                       "d": rng.normal(0, .1, so)})
    return params


DIMS = [(2, 4, 3, 3), (3, 3, 3, 3), (3, 3, 1, 2)]


def loss_of(params, xg, xs, tg, ts, B, G, slope=0.1):
    yg, ys, _ = R.forward(params, xg, xs, B, G, slope)
    return 0.5 * np.sum((yg - tg) ** 2) + 0.5 * np.sum((ys - ts) ** 2)


def test_reference_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    B, G, H, W = 2, 3, 5, 6
    params = small_net(rng, DIMS)
    xg, xs = rng.normal(size=(B * G, 2, H, W)), rng.normal(size=(B, 4, H, W))
    tg, ts = rng.normal(size=(B * G, 1, H, W)), rng.normal(size=(B, 2, H, W))
    yg, ys, cache = R.forward(params, xg, xs, B, G, 0.1)
    grads = R.backward(params, cache, yg - tg, ys - ts, B, G, 0.1)
    eps = 1e-6
    for l in range(len(DIMS)):
        for k in ("A", "B", "C", "D", "E", "a", "d"):
            flat = params[l][k].reshape(-1)
            for idx in rng.choice(flat.size, size=min(3, flat.size), replace=False):
                old = flat[idx]
                flat[idx] = old + eps
                lp = loss_of(params, xg, xs, tg, ts, B, G)
                flat[idx] = old - eps
                lm = loss_of(params, xg, xs, tg, ts, B, G)
                flat[idx] = old
                fd = (lp - lm) / (2 * eps)
                an = grads[l][k].reshape(-1)[idx]
                assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (l, k, fd, an)


def test_reference_is_grain_permutation_equivariant():
    rng = np.random.default_rng(1)
    B, G, H, W = 1, 4, 6, 6
    params = small_net(rng, DIMS)
    xg, xs = rng.normal(size=(B * G, 2, H, W)), rng.normal(size=(B, 4, H, W))
    perm = np.array([2, 0, 3, 1])
    yg, ys, _ = R.forward(params, xg, xs, B, G, 0.1)
    yg2, ys2, _ = R.forward(params, xg[perm], xs, B, G, 0.1)
    assert np.allclose(yg2, yg[perm], atol=1e-12)
    assert np.allclose(ys2, ys, atol=1e-12)


def test_adam_reference_first_step_moves_by_lr():
    p, g = np.array([1.0, -2.0]), np.array([0.5, -3.0])
    p1, m, v = R.adam(p, g, np.zeros(2), np.zeros(2), 1e-3, 0.9, 0.999, 1e-8, 1)
    # bias-corrected first step: m_hat / sqrt(v_hat) = sign(g)
    assert np.allclose(p - p1, 1e-3 * np.sign(g), rtol=1e-6)


def small_net3(rng, dims):
    params = []
    for (cg, cs, go, so) in dims:
        w = lambda co, ci: rng.normal(0, .2, (3, co, ci, 3, 3))
        params.append({"A": w(go, cg), "B": w(go, cg), "C": w(go, cs), "D": w(so, cs), "E": w(so, cg),
                       "a": rng.normal(0, .1, go), "d": rng.normal(0, .1, so)})
    return params


def test_reference_conv3x3x3_is_the_27_tap_convolution():
    """The depth-offset decomposition equals a direct 27-tap correlation with
    zero padding (x [N][D][C][H][W], w3[dz + 1][co][ci][ky][kx])."""
    rng = np.random.default_rng(7)
    N, D, Cin, Cout, H, W = 2, 4, 3, 2, 5, 6
    x, w3, b = rng.normal(size=(N, D, Cin, H, W)), rng.normal(size=(3, Cout, Cin, 3, 3)), rng.normal(size=Cout)
    xp = np.zeros((N, D + 2, Cin, H + 2, W + 2))
    xp[:, 1:-1, :, 1:-1, 1:-1] = x
    ref = np.zeros((N, D, Cout, H, W)) + b[None, None, :, None, None]
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                ref += np.einsum("oc,ndchw->ndohw", w3[kz, :, :, ky, kx], xp[:, kz:kz + D, :, ky:ky + H, kx:kx + W])
    assert np.allclose(R.conv3x3x3(x, w3, b), ref, atol=1e-12)


def test_reference_3d_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    B, G, D, H, W = 1, 2, 3, 4, 4
    dims = [(2, 4, 3, 3), (3, 3, 1, 2)]
    params = small_net3(rng, dims)
    xg, xs = rng.normal(size=(B * G, D, 2, H, W)), rng.normal(size=(B, D, 4, H, W))
    tg, ts = rng.normal(size=(B * G, D, 1, H, W)), rng.normal(size=(B, D, 2, H, W))
    yg, ys, cache = R.forward(params, xg, xs, B, G, 0.1)
    grads = R.backward(params, cache, yg - tg, ys - ts, B, G, 0.1)
    eps = 1e-6
    for l in range(len(dims)):
        for k in ("A", "B", "C", "D", "E", "a", "d"):
            flat = params[l][k].reshape(-1)
            for idx in rng.choice(flat.size, size=min(3, flat.size), replace=False):
                old = flat[idx]
                flat[idx] = old + eps
                lp = loss_of(params, xg, xs, tg, ts, B, G)
                flat[idx] = old - eps
                lm = loss_of(params, xg, xs, tg, ts, B, G)
                flat[idx] = old
                fd = (lp - lm) / (2 * eps)
                an = grads[l][k].reshape(-1)[idx]
                assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (l, k, fd, an)
