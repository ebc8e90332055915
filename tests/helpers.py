"""Shared helpers of the test-suite: random sintering states, parity metrics."""
import itertools

import numpy as np

from oracle import oracle as O


def n_nodes(dim, cells):
    n = 1
    for d in range(dim):
        n *= cells[d] + 1
    return n


def oracle_mesh(dim, cells, h=(1.0, 1.0, 1.0)):
    return O.make_mesh(dim, list(cells) + [0] * (3 - len(cells)), h)


def random_state(dim, cells, G, seed, smooth=True):
    """A (C, N) state with c, eta in [0, 1] and mu in [-1, 1].  With smooth=True
    the fields are sums of a few random Fourier modes (realistic interfaces, all
    mobility branches active) plus small noise; otherwise i.i.d. uniform."""
    rng = np.random.default_rng(seed)
    C = G + 2
    shape = [cells[d] + 1 for d in range(dim)]
    N = int(np.prod(shape))
    if not smooth:
        u = rng.uniform(0.0, 1.0, (C, N))
        u[1] = rng.uniform(-1.0, 1.0, N)
        return u
    axes = np.meshgrid(*[np.linspace(0, 1, s) for s in shape], indexing="ij")
    u = np.zeros((C, N))
    for b in range(C):
        f = np.zeros(shape)
        for _ in range(3):
            k = rng.integers(1, 4, dim)
            ph = rng.uniform(0, 2 * np.pi, dim)
            term = np.ones(shape)
            for d in range(dim):
                term = term * np.cos(np.pi * k[d] * axes[d] + ph[d])
            f += rng.uniform(0.3, 1.0) * term
        f = 0.5 + 0.5 * f / 3.0 + rng.uniform(-0.02, 0.02, shape)
        if b == 1:
            f = 2.0 * f - 1.0
        # numpy meshgrid 'ij' has x first; our node order is x fastest
        u[b] = np.transpose(f).ravel()
    return u


def block_rel_err(ours, ref):
    """max over blocks of |ours_b - ref_b|_2 / |ref_b|_2 (absolute if ref_b == 0)."""
    errs = []
    for b in range(ref.shape[0]):
        nr = np.linalg.norm(ref[b])
        ne = np.linalg.norm(ours[b] - ref[b])
        errs.append(ne / nr if nr > 0 else ne)
    return max(errs)


def particle_state(dim, cells, G, seed, width=1.0):
    """A (C, N) packing state whose grains are localised: every grain owns one
    or two round particles (tanh profile of the given interface width), c is
    the largest eta, mu a smooth random field.  Far from a particle its eta
    decays to ~1e-10 and below, so grain cut-off masks vary from cell to cell.
    Each eta carries a smooth 5 % modulation of its own (keeping eta < 1, where
    the clamp of the interpolation function is inactive): without it the
    plateaus where particles of two grains overlap have gradients of ~1e-9, and
    the direction of grad eta_i - grad eta_j that the tensorial mobility's
    grain-boundary projector needs is rounding noise there (an ill-conditioned
    state, not a test of the operator)."""
    rng = np.random.default_rng(seed)
    shape = [cells[d] + 1 for d in range(dim)]
    axes = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij")
    C = G + 2
    u = np.zeros((C, int(np.prod(shape))))
    etas = []
    for g in range(G):
        eta = np.zeros(shape)
        for _ in range(int(rng.integers(1, 3))):
            ctr = [rng.uniform(0, cells[d]) for d in range(dim)]
            R = rng.uniform(1.0, 0.3 * min(cells[:dim]) + 1.0)
            r = np.sqrt(sum((axes[d] - ctr[d]) ** 2 for d in range(dim)))
            eta = np.maximum(eta, 0.5 * (1.0 - np.tanh((r - R) / (0.5 * width))))
        k = rng.integers(1, 4, dim)
        ph = rng.uniform(0, 2 * np.pi)
        eta = eta * (0.95 + 0.05 * np.cos(sum(np.pi * k[d] * axes[d] / max(1, cells[d]) for d in range(dim)) + ph))
        etas.append(eta)
        u[2 + g] = np.transpose(eta).ravel()
    u[0] = np.transpose(np.max(etas, axis=0)).ravel()
    mu = np.zeros(shape)
    for _ in range(3):
        k = rng.integers(1, 4, dim)
        ph = rng.uniform(0, 2 * np.pi, dim)
        term = np.ones(shape)
        for d in range(dim):
            term = term * np.cos(np.pi * k[d] * axes[d] / max(1, cells[d]) + ph[d])
        mu += rng.uniform(0.3, 1.0) * term
    u[1] = np.transpose(mu).ravel() / 3.0
    return u


def grain_mask_numpy(dim, cells, G, u, tol):
    """The cut-off rule restated in numpy: bit b set on a cell when the largest
    |eta_b| over its nodes exceeds tol (cells x fastest)."""
    shape = [cells[d] + 1 for d in range(dim)]
    mask = np.zeros([cells[d] for d in range(dim)], dtype=np.uint16)
    for b in range(G):
        eta = np.abs(u[2 + b].reshape(list(reversed(shape))).T)  # index [x, y, (z)]
        m = np.zeros([cells[d] for d in range(dim)])
        for corner in range(1 << dim):
            sl = tuple(slice((corner >> d) & 1, ((corner >> d) & 1) + cells[d]) for d in range(dim))
            m = np.maximum(m, eta[sl])
        mask |= ((m > tol).astype(np.uint16) << b)
    return np.transpose(mask).ravel()


def tracker_golden_field(g):
    """The nodal field of grain_tracker_elliptical.cc: 1 inside the ellipse or
    the circle, 0 elsewhere, on the golden's uniform mesh (nodes x fastest).
    Returns (dim, cells, h, origin, eta)."""
    mesh = g["mesh"]
    cells = mesh["cells"]
    h = [(mesh["upper"][d] - mesh["lower"][d]) / cells[d] for d in range(2)]
    xs = mesh["lower"][0] + np.arange(cells[0] + 1) * h[0]
    ys = mesh["lower"][1] + np.arange(cells[1] + 1) * h[1]
    X, Y = np.meshgrid(xs, ys, indexing="xy")  # rows = y: x fastest when raveled
    e, c = g["ellipse"], g["circle"]
    q = ((X - e["center"][0]) / e["semi_axes"][0]) ** 2 + ((Y - e["center"][1]) / e["semi_axes"][1]) ** 2
    in_e = q <= 1.0 if e["inclusive"] else q < 1.0
    r = np.sqrt((X - c["center"][0]) ** 2 + (Y - c["center"][1]) ** 2)
    in_c = r <= c["radius"] if c["inclusive"] else r < c["radius"]
    return 2, cells, h, mesh["lower"], np.where(in_e | in_c, 1.0, 0.0).ravel()


def advection_data(dim, cells, G, seed, n_seg_per_grain=2, scale=1.0):
    """Random segment assignment (-1 on about a third of the cells) and random
    segment velocities/centers."""
    rng = np.random.default_rng(seed)
    n_cells = int(np.prod(cells))
    S = G * n_seg_per_grain
    seg = np.full((G, n_cells), -1, dtype=np.int32)
    for b in range(G):
        pick = rng.integers(0, n_seg_per_grain, n_cells) + b * n_seg_per_grain
        seg[b] = np.where(rng.uniform(size=n_cells) < 0.67, pick, -1)
    data = np.zeros((S, 9))
    data[:, 0:3] = scale * rng.normal(size=(S, 3))
    data[:, 3:6] = 0.2 * scale * rng.normal(size=(S, 3))
    data[:, 6:9] = rng.uniform(0, 4, size=(S, 3))
    if dim == 2:
        data[:, 2] = 0.0
    return seg, data


def max_speed(dim, cells, h, origin, seg, data, mask=None):
    """Largest |v| over the quadrature points of every (cell, grain) with a segment."""
    n_cells = int(np.prod(cells))
    idx = np.arange(n_cells)
    co = np.stack([idx % cells[0], (idx // cells[0]) % cells[1],
                   idx // (cells[0] * cells[1]) if dim == 3 else np.zeros_like(idx)], axis=1)
    vmax = 0.0
    for b in range(seg.shape[0]):
        sel = seg[b] >= 0
        if mask is not None:
            sel &= ((mask >> b) & 1).astype(bool)
        s = seg[b, sel]
        for qb in itertools.product((0, 1), repeat=dim):
            x = np.zeros((s.size, 3))
            for d in range(dim):
                x[:, d] = origin[d] + (co[sel, d] + (0.5 + (qb[d] - 0.5) / np.sqrt(3.0))) * h[d]
            r = x - data[s, 6:9]
            if dim == 2:
                r[:, 2] = 0.0
            v = data[s, 0:3] + np.cross(data[s, 3:6], r)
            if dim == 2:
                v[:, 2] = 0.0
            if v.size:
                vmax = max(vmax, float(np.sqrt((v ** 2).sum(axis=1)).max()))
    return vmax


def tracker_periodic_golden_fields(g):
    """Nodal fields of the order parameters of the grain_tracker_advection_periodic
    golden: cosine-interface discs (1 inside R - w/2, (1 + cos(pi (r - R + w/2)
    / w)) / 2 across the interface of width w, 0 outside), the largest over the
    particles of each order parameter.  Returns dim, cells, h, origin, fields."""
    mesh = g["mesh"]
    cells = mesh["cells"]
    h = [(mesh["upper"][d] - mesh["lower"][d]) / cells[d] for d in range(2)]
    X, Y = np.meshgrid(mesh["lower"][0] + np.arange(cells[0] + 1) * h[0],
                       mesh["lower"][1] + np.arange(cells[1] + 1) * h[1])
    w = g["interface_width"]
    n_ops = 1 + max(p[3] for p in g["particles"])
    fields = [np.zeros_like(X) for _ in range(n_ops)]
    for cx, cy, R, op in g["particles"]:
        r = np.hypot(X - cx, Y - cy)
        v = np.where(r <= R - w / 2, 1.0, np.where(r < R + w / 2, (1 + np.cos((r - R + w / 2) / w * np.pi)) / 2, 0.0))
        fields[op] = np.maximum(fields[op], v)
    return 2, cells, h, mesh["lower"], [f.ravel() for f in fields]


def group_grains(op_index, props, groups, dim=2):
    """Grains of one order parameter: periodic groups become one grain of
    several segments, the other particles one grain each.  props rows:
    measure, center[dim], radius, max value.  Returns [(op, sorted segments
    [center..., radius, max])]."""
    seg = [list(p[1:1 + dim]) + [p[1 + dim], p[2 + dim]] for p in props]
    by_group, grains = {}, []
    for i, gid in enumerate(groups):
        if gid < 0:
            grains.append((op_index, [seg[i]]))
        else:
            by_group.setdefault(gid, []).append(seg[i])
    grains += [(op_index, sorted(v)) for v in by_group.values()]
    return grains


def grains_agree(ours, ref, digits):
    """Same multiset of (op, segments) to `digits` significant digits."""
    key = lambda gr: (gr[0], len(gr[1]), gr[1][0][0], gr[1][0][1])  # noqa: E731
    ours, ref = sorted(ours, key=key), sorted(ref, key=key)
    if len(ours) != len(ref):
        return False
    rtol = 0.5 * 10.0 ** (1 - digits)
    for (oa, sa), (ob, sb) in zip(ours, ref):
        if oa != ob or len(sa) != len(sb):
            return False
        if not all(np.allclose(x, y, rtol=rtol, atol=0) for x, y in zip(sa, sb)):
            return False
    return True
