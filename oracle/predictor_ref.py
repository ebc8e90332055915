"""NumPy reference of the learned-guess network (test infrastructure only).

Float64 restatement of the grain-permutation-equivariant conv net whose
forward, backward and Adam kernels live in the CUDA library; the tests
compare the CUDA results with these and check the analytic gradients against
central finite differences.  Layout NCHW; grain streams of sample b are batch
entries b * G + i.
"""
import numpy as np


def conv3x3(x, w, b=None):
    """x [N][Cin][H][W], w [Cout][Cin][3][3] -> [N][Cout][H][W] (zero padding)."""
    N, Cin, H, W = x.shape
    xp = np.zeros((N, Cin, H + 2, W + 2))
    xp[:, :, 1:-1, 1:-1] = x
    out = np.zeros((N, w.shape[0], H, W))
    for ky in range(3):
        for kx in range(3):
            out += np.einsum("oc,nchw->nohw", w[:, :, ky, kx], xp[:, :, ky:ky + H, kx:kx + W])
    if b is not None:
        out += b[None, :, None, None]
    return out


def conv3x3_input_grad(dout, w):
    """d/dx of sum(dout * conv3x3(x, w))."""
    wT = np.transpose(w[:, :, ::-1, ::-1], (1, 0, 2, 3))
    return conv3x3(dout, wT)


def conv3x3_weight_grad(x, dout):
    N, Cin, H, W = x.shape
    xp = np.zeros((N, Cin, H + 2, W + 2))
    xp[:, :, 1:-1, 1:-1] = x
    dw = np.zeros((dout.shape[1], Cin, 3, 3))
    for ky in range(3):
        for kx in range(3):
            dw[:, :, ky, kx] = np.einsum("nohw,nchw->oc", dout, xp[:, :, ky:ky + H, kx:kx + W])
    return dw, dout.sum(axis=(0, 2, 3))


def leaky(x, s):
    return np.where(x > 0, x, s * x)


def leaky_grad(x, s):
    return np.where(x > 0, 1.0, s)


def grain_sum(h, B, G):
    return h.reshape(B, G, *h.shape[1:]).sum(axis=1)


def bcast(Q, G):
    return np.repeat(Q, G, axis=0)


def forward(params, xg, xs, B, G, slope):
    """params: list of dicts A..E, a, d per layer; returns outputs and cache."""
    hg, hs, cache = xg, xs, []
    n = len(params)
    for l, w in enumerate(params):
        P = grain_sum(hg, B, G)
        Zg = conv3x3(hg, w["A"], w["a"]) + bcast(conv3x3(P, w["B"]) + conv3x3(hs, w["C"]), G)
        Zs = conv3x3(hs, w["D"], w["d"]) + conv3x3(P, w["E"])
        cache.append((hg, hs, P, Zg, Zs))
        if l < n - 1:
            hg, hs = leaky(Zg, slope), leaky(Zs, slope)
        else:
            hg, hs = Zg, Zs
    return hg, hs, cache


def backward(params, cache, dyg, dys, B, G, slope):
    grads = [dict() for _ in params]
    dZg, dZs = dyg, dys
    n = len(params)
    for l in reversed(range(n)):
        hg, hs, P, Zg, Zs = cache[l]
        w = params[l]
        if l < n - 1:
            dZg = dZg * leaky_grad(Zg, slope)
            dZs = dZs * leaky_grad(Zs, slope)
        dQ = grain_sum(dZg, B, G)
        grads[l]["A"], grads[l]["a"] = conv3x3_weight_grad(hg, dZg)
        grads[l]["B"], _ = conv3x3_weight_grad(P, dQ)
        grads[l]["C"], _ = conv3x3_weight_grad(hs, dQ)
        grads[l]["D"], grads[l]["d"] = conv3x3_weight_grad(hs, dZs)
        grads[l]["E"], _ = conv3x3_weight_grad(P, dZs)
        dP = conv3x3_input_grad(dQ, w["B"]) + conv3x3_input_grad(dZs, w["E"])
        dhg = conv3x3_input_grad(dZg, w["A"]) + bcast(dP, G)
        dhs = conv3x3_input_grad(dQ, w["C"]) + conv3x3_input_grad(dZs, w["D"])
        dZg, dZs = dhg, dhs
    return grads


def adam(p, g, m, v, lr, b1, b2, eps, t):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return p, m, v
