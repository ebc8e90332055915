"""NumPy reference of the learned-guess network (test infrastructure only).

Float64 restatement of the grain-permutation-equivariant conv net whose
forward, backward and Adam kernels live in the CUDA library; the tests
compare the CUDA results with these and check the analytic gradients against
central finite differences.  Layout NCHW; grain streams of sample b are batch
entries b * G + i.  3D: layout [N][D][C][H][W] (depth-major, no padding
slices here) and weights [3][Cout][Cin][3][3], index 0 multiplying the slice
below; the 3x3x3 convolution is restated as the sum over depth offsets of
3x3 convolutions.
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


def conv3x3x3(x, w3, b=None):
    """x [N][D][Cin][H][W], w3 [3][Cout][Cin][3][3] -> [N][D][Cout][H][W] (zero padding)."""
    N, D = x.shape[:2]
    out = np.zeros((N, D, w3.shape[1]) + x.shape[3:])
    for j, dz in enumerate((-1, 0, 1)):
        for z in range(D):
            if 0 <= z + dz < D:
                out[:, z] += conv3x3(x[:, z + dz], w3[j])
    if b is not None:
        out += b[None, None, :, None, None]
    return out


def conv3x3x3_input_grad(dout, w3):
    """d/dx of sum(dout * conv3x3x3(x, w3))."""
    N, D = dout.shape[:2]
    din = np.zeros((N, D, w3.shape[2]) + dout.shape[3:])
    for j, dz in enumerate((-1, 0, 1)):
        for z in range(D):
            if 0 <= z + dz < D:
                din[:, z + dz] += conv3x3_input_grad(dout[:, z], w3[j])
    return din


def conv3x3x3_weight_grad(x, dout):
    N, D = x.shape[:2]
    dw = np.zeros((3, dout.shape[2], x.shape[2], 3, 3))
    for j, dz in enumerate((-1, 0, 1)):
        for z in range(D):
            if 0 <= z + dz < D:
                dw[j] += conv3x3_weight_grad(x[:, z + dz], dout[:, z])[0]
    return dw, dout.sum(axis=(0, 1, 3, 4))


def _conv(x, w, b=None):
    return conv3x3(x, w, b) if w.ndim == 4 else conv3x3x3(x, w, b)


def _input_grad(dout, w):
    return conv3x3_input_grad(dout, w) if w.ndim == 4 else conv3x3x3_input_grad(dout, w)


def _weight_grad(x, dout):
    return conv3x3_weight_grad(x, dout) if x.ndim == 4 else conv3x3x3_weight_grad(x, dout)


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
        Zg = _conv(hg, w["A"], w["a"]) + bcast(_conv(P, w["B"]) + _conv(hs, w["C"]), G)
        Zs = _conv(hs, w["D"], w["d"]) + _conv(P, w["E"])
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
        grads[l]["A"], grads[l]["a"] = _weight_grad(hg, dZg)
        grads[l]["B"], _ = _weight_grad(P, dQ)
        grads[l]["C"], _ = _weight_grad(hs, dQ)
        grads[l]["D"], grads[l]["d"] = _weight_grad(hs, dZs)
        grads[l]["E"], _ = _weight_grad(P, dZs)
        dP = _input_grad(dQ, w["B"]) + _input_grad(dZs, w["E"])
        dhg = _input_grad(dZg, w["A"]) + bcast(dP, G)
        dhs = _input_grad(dQ, w["C"]) + _input_grad(dZs, w["D"])
        dZg, dZs = dhg, dhs
    return grads


def adam(p, g, m, v, lr, b1, b2, eps, t):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return p, m, v
