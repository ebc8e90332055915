"""Advection (rigid-body motion of the grains) in the CPU oracle (no GPU).

With AdvectionMechanism enabled, the residual and the Jacobian of
SinteringOperatorGeneric gain, per grain i with a velocity on the cell,
  c row:     -(v_i c,     grad phi)   (operator_sintering_generic.h:1015-1036)
  eta_i row: -(v_i eta_i, grad phi)   (the J v form at :167-177)
with v_i = v_t + w x (x_q - center) of the grain segment the cell belongs to
(AdvectionVelocityData::get_velocity, sintering/advection.h:247-263, with the
2D cross product of :105-113).  These tests pin the oracle's restatement
against an independent numpy quadrature, check that the terms conserve mass
and are linear in the velocities, and check the Jacobian by central
differences at frozen velocities (as the reference's tangent tests do).
"""
import itertools

import numpy as np
import pytest

from helpers import advection_data, max_speed, oracle_mesh, random_state
from oracle import oracle as O

GP = (0.5 - 0.5 / np.sqrt(3.0), 0.5 + 0.5 / np.sqrt(3.0))


def numpy_advection(dim, cells, h, origin, u, seg, data):
    """-(v_i c, grad phi) and -(v_i eta_i, grad phi), assembled cell by cell
    with 2-point Gauss quadrature (plain loops, small meshes only)."""
    G = u.shape[0] - 2
    nn = [c + 1 for c in cells]
    out = np.zeros_like(u)
    corners = list(itertools.product((0, 1), repeat=dim))  # corners[a][d] = bit d
    for cc in itertools.product(*[range(c) for c in reversed(cells)]):
        cc = tuple(reversed(cc))  # x fastest
        cell = sum(cc[d] * int(np.prod(cells[:d])) for d in range(dim))
        nodes = [sum((cc[d] + a[d]) * int(np.prod(nn[:d])) for d in range(dim)) for a in corners]
        for qb in itertools.product((0, 1), repeat=dim):
            xi = [GP[qb[d]] for d in range(dim)]
            w = np.prod([h[d] for d in range(dim)]) / 2 ** dim
            N = np.array([np.prod([xi[d] if a[d] else 1 - xi[d] for d in range(dim)]) for a in corners])
            dN = np.zeros((len(corners), dim))
            for k, a in enumerate(corners):
                for d in range(dim):
                    f = (1.0 if a[d] else -1.0) / h[d]
                    for e in range(dim):
                        if e != d:
                            f *= xi[e] if a[e] else 1 - xi[e]
                    dN[k, d] = f
            x = np.array([origin[d] + (cc[d] + xi[d]) * h[d] for d in range(dim)] + [0.0] * (3 - dim))
            for i in range(G):
                s = seg[i, cell]
                if s < 0:
                    continue
                r = x - data[s, 6:9]
                if dim == 2:
                    r[2] = 0.0
                v = data[s, 0:3] + np.cross(data[s, 3:6], r)
                v = v[:dim]
                cq = N @ u[0, nodes]
                eq = N @ u[2 + i, nodes]
                out[0, nodes] -= w * cq * (dN @ v)
                out[2 + i, nodes] -= w * eq * (dN @ v)
    return out


CASES = [(2, (6, 5), 3, False), (2, (7, 4), 2, True), (3, (4, 3, 3), 3, False), (3, (3, 4, 2), 2, True)]


@pytest.mark.parametrize("dim,cells,G,tens", CASES)
def test_matches_independent_quadrature(dim, cells, G, tens):
    h = (0.7, 1.3, 0.9)
    origin = (1.5, -2.0, 0.25)
    om, p = O.make_mesh(dim, list(cells) + [0] * (3 - dim), h), O.make_params(G, tensorial=tens)
    u = random_state(dim, cells, G, seed=4)
    seg, data = advection_data(dim, cells, G, seed=5)
    T = O.make_time(10.0, 1.0, [-10.0])
    adv = (seg, data, origin)
    diff = O.residual(om, p, T, u, [u], 2, advection=adv) - O.residual(om, p, T, u, [u], 2)
    ref = numpy_advection(dim, cells, h, origin, u, seg, data)
    assert np.allclose(diff, ref, rtol=1e-11, atol=1e-13 * np.abs(ref).max())
    # the J v terms are the same bilinear form in the direction
    src = random_state(dim, cells, G, seed=6, smooth=False) - 0.5
    jd = O.jvp(om, p, T, u, src, advection=adv) - O.jvp(om, p, T, u, src)
    ref = numpy_advection(dim, cells, h, origin, src, seg, data)
    assert np.allclose(jd, ref, rtol=1e-11, atol=1e-13 * np.abs(ref).max())


@pytest.mark.parametrize("dim,cells,G,tens", CASES)
def test_conservative_and_linear_in_velocity(dim, cells, G, tens):
    om, p = oracle_mesh(dim, cells), O.make_params(G, tensorial=tens)
    u = random_state(dim, cells, G, seed=7)
    seg, data = advection_data(dim, cells, G, seed=8)
    T = O.make_time(10.0, 1.0, [-10.0])
    base = O.residual(om, p, T, u, [u], 2)
    d1 = O.residual(om, p, T, u, [u], 2, advection=(seg, data, (0, 0, 0))) - base
    # the test functions sum to one: a flux term adds nothing to the total
    assert np.abs(d1.sum(axis=1)).max() < 1e-12 * np.abs(d1).max()
    data2 = data.copy()
    data2[:, 0:6] *= 2.5
    d2 = O.residual(om, p, T, u, [u], 2, advection=(seg, data2, (0, 0, 0))) - base
    assert np.allclose(d2, 2.5 * d1, rtol=1e-10, atol=1e-13 * np.abs(d1).max())
    # no segment anywhere is no advection at all
    none = np.full_like(seg, -1)
    assert np.array_equal(O.residual(om, p, T, u, [u], 2, advection=(none, data, (0, 0, 0))), base)


@pytest.mark.parametrize("dim,cells,G", [(2, (9, 7), 3), (3, (5, 4, 4), 3)])
def test_jacobian_by_central_differences(dim, cells, G):
    om, p = oracle_mesh(dim, cells), O.make_params(G, tensorial=False)
    u = random_state(dim, cells, G, seed=9)
    src = random_state(dim, cells, G, seed=10, smooth=False) - 0.5
    seg, data = advection_data(dim, cells, G, seed=11)
    adv = (seg, data, (0.5, 0.5, 0.5))
    T = O.make_time(10.0, 1.0, [-10.0])
    eps = 1e-6
    fd = (O.residual(om, p, T, u + eps * src, [u], 2, advection=adv)
          - O.residual(om, p, T, u - eps * src, [u], 2, advection=adv)) / (2 * eps)
    jv = O.jvp(om, p, T, u, src, advection=adv)
    scale = np.abs(jv).max(axis=1, keepdims=True)
    assert (np.abs(fd - jv) / scale).max() < 1e-6


def test_mask_and_advection_together():
    """With the grain cut-off a grain absent from a cell has no advection
    there either (AdvectionVelocityData::has_velocity through the relevant-grain
    map, sintering/advection.h:231-245)."""
    dim, cells, G = 2, (8, 6), 3
    om, p = oracle_mesh(dim, cells), O.make_params(G)
    u = random_state(dim, cells, G, seed=12)
    seg, data = advection_data(dim, cells, G, seed=13)
    T = O.make_time(10.0, 1.0, [-10.0])
    rng = np.random.default_rng(14)
    mask = rng.integers(0, 1 << G, int(np.prod(cells))).astype(np.uint16)
    seg_m = seg.copy()
    for b in range(G):
        seg_m[b, (mask >> b) & 1 == 0] = -1
    a = O.residual(om, p, T, u, [u], 2, mask=mask, advection=(seg, data, (0, 0, 0)))
    b_ = O.residual(om, p, T, u, [u], 2, mask=mask, advection=(seg_m, data, (0, 0, 0)))
    assert np.array_equal(a, b_)


# --- the advection mechanism: forces, torques, volumes and the velocity table


def test_velocities_match_golden(goldens):
    """AdvectionMechanism's velocities (advection_mechanism_data golden):
    three segments with volume, force, torque and center, velocities at the
    cell barycenters of a 4 x 4 mesh of [0, 1]^2, mt = mr = 1."""
    g = goldens["advection_mechanism_data"]
    nc = g["n_comp_volume_force_torque"]
    vft = np.array(g["grains_data"]).reshape(-1, nc)
    S = vft.shape[0]
    centers = np.zeros((S, 3))
    centers[:, :2] = np.array(g["grain_center"]).reshape(S, 2)
    table = O.advection_velocities(2, vft, centers, g["mt"], g["mr"])
    lanes = g["lanes"]
    for batch in g["batches"]:
        # op 0: center (0, 0) and mr torque / volume = 1, so its rotation
        # velocity (-y, x) gives the lanes' evaluation points
        rot0 = np.array(batch[0]["rot_vel"]).reshape(2, lanes)
        pts = np.stack([rot0[1], -rot0[0]], axis=1)
        assert np.allclose(pts / g["h"][0] % 1.0, 0.5, atol=1e-5)  # cell barycenters
        for entry in batch:
            s = entry["op"]
            assert entry["has_velocity"] == 1
            vt = np.tile(table[s, 0:2], (lanes, 1))
            r = pts - table[s, 6:8]
            vr = table[s, 5] * np.stack([-r[:, 1], r[:, 0]], axis=1)
            for ours, key in ((vt, "trans_vel"), (vr, "rot_vel"), (vt + vr, "tot_vel")):
                ref = np.array(entry[key]).reshape(2, lanes).T
                assert np.allclose(ours, ref, rtol=1e-5, atol=1e-6), (s, key, ours, ref)


def numpy_forces(dim, cells, h, origin, u, seg, centers, k, cgb, ceq, smoothening, mask=None):
    G = u.shape[0] - 2
    nn = [c + 1 for c in cells]
    nt = 3 if dim == 3 else 1
    out = np.zeros((centers.shape[0], 1 + dim + nt))
    corners = list(itertools.product((0, 1), repeat=dim))
    for cc in itertools.product(*[range(c) for c in reversed(cells)]):
        cc = tuple(reversed(cc))
        cell = sum(cc[d] * int(np.prod(cells[:d])) for d in range(dim))
        rel = [b for b in range(G) if mask is None or (int(mask[cell]) >> b) & 1]
        nodes = [sum((cc[d] + a[d]) * int(np.prod(nn[:d])) for d in range(dim)) for a in corners]
        for qb in itertools.product((0, 1), repeat=dim):
            xi = [GP[qb[d]] for d in range(dim)]
            w = np.prod([h[d] for d in range(dim)]) / 2 ** dim
            N = np.array([np.prod([xi[d] if a[d] else 1 - xi[d] for d in range(dim)]) for a in corners])
            dN = np.zeros((len(corners), dim))
            for kk, a in enumerate(corners):
                for d in range(dim):
                    f = (1.0 if a[d] else -1.0) / h[d]
                    for e in range(dim):
                        if e != d:
                            f *= xi[e] if a[e] else 1 - xi[e]
                    dN[kk, d] = f
            x = np.array([origin[d] + (cc[d] + xi[d]) * h[d] for d in range(dim)])
            val = u[:, nodes] @ N
            grad = u[:, nodes] @ dN
            for i in rel:
                s = seg[i, cell]
                if s < 0:
                    continue
                r = x - centers[s, :dim]
                out[s, 0] += w * val[2 + i]
                for j in rel:
                    if j == i:
                        continue
                    p = val[2 + i] * val[2 + j]
                    if cgb > 0:
                        f = 1 / (1 + np.exp(-smoothening * (p - cgb))) if smoothening > 0 else float(p > cgb)
                    else:
                        f = 4 * p
                    dF = k * (val[0] - ceq) * f * (grad[2 + i] - grad[2 + j])
                    out[s, 1:1 + dim] += w * dF
                    if dim == 3:
                        out[s, 4:7] += w * np.cross(r, dF)
                    else:
                        out[s, 3] += w * (r[1] * dF[0] - r[0] * dF[1])  # tensor.h:62-66
    return out


@pytest.mark.parametrize("dim,cells,G", [(2, (7, 6), 3), (3, (4, 3, 3), 3)])
@pytest.mark.parametrize("cgb,smoothening", [(0.0, 0.0), (0.14, 0.0), (0.14, 40.0)])
def test_forces_match_independent_quadrature(dim, cells, G, cgb, smoothening):
    h = (0.7, 1.3, 0.9)
    origin = (1.5, -2.0, 0.25)
    om, p = O.make_mesh(dim, list(cells) + [0] * (3 - dim), h), O.make_params(G)
    u = random_state(dim, cells, G, seed=21)
    seg, data = advection_data(dim, cells, G, seed=22)
    centers = data[:, 6:9]
    ref = numpy_forces(dim, cells, h, origin, u, seg, centers, 2.5, cgb, 0.9, smoothening)
    got = O.advection_forces(om, p, u, seg, centers, origin, 2.5, cgb, 0.9, smoothening)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-13 * np.abs(ref).max())
    assert np.abs(ref[:, 1:]).max() > 1e-3  # non-trivial forces
    # under the grain cut-off only the relevant grains act
    mask = np.random.default_rng(23).integers(0, 1 << G, int(np.prod(cells))).astype(np.uint16)
    ref_m = numpy_forces(dim, cells, h, origin, u, seg, centers, 2.5, cgb, 0.9, smoothening, mask)
    got_m = O.advection_forces(om, p, u, seg, centers, origin, 2.5, cgb, 0.9, smoothening, mask=mask)
    assert np.allclose(got_m, ref_m, rtol=1e-12, atol=1e-13 * np.abs(ref_m).max())


@pytest.mark.parametrize("dim,cells", [(2, (12, 10)), (3, (6, 5, 5))])
def test_forces_balance(dim, cells):
    """With every grain one segment over the whole mesh, the pair forces
    cancel (dF_ji = -dF_ij with the symmetric 4 eta_i eta_j weight), and so do
    the torques about a common center."""
    G = 3
    om, p = oracle_mesh(dim, cells), O.make_params(G)
    u = random_state(dim, cells, G, seed=24)
    n_cells = int(np.prod(cells))
    seg = np.repeat(np.arange(G, dtype=np.int32)[:, None], n_cells, axis=1)
    centers = np.tile([1.0, 2.0, 0.5], (G, 1))
    f = O.advection_forces(om, p, u, seg, centers, (0, 0, 0), 3.0, 0.0, 0.8, 0.0)
    scale = np.abs(f[:, 1:]).max()
    assert scale > 1e-3
    assert np.abs(f[:, 1:].sum(axis=0)).max() < 1e-12 * scale
    # volumes: the integral of each eta (Q1 basis functions integrate to the trapezoidal weights)
    w = np.ones(1)
    for d in range(dim):
        wd = np.ones(cells[d] + 1)
        wd[[0, -1]] = 0.5
        w = np.kron(wd, w)
    assert np.allclose(f[:, 0], u[2:] @ w, rtol=1e-13)


@pytest.mark.parametrize("dim,cells,G", [(2, (9, 7), 3), (3, (5, 4, 4), 3)])
def test_courant_check(dim, cells, G):
    """CFLChecker::check_courant: violated exactly when |v| dt reaches the
    cell diameter somewhere a relevant grain moves."""
    h = (0.7, 1.3, 0.9)
    om, p = O.make_mesh(dim, list(cells) + [0] * (3 - dim), h), O.make_params(G)
    seg, data = advection_data(dim, cells, G, seed=31)
    adv = (seg, data, (0.5, -1.0, 0.0))
    diam = np.sqrt(sum(h[d] ** 2 for d in range(dim)))
    dt_crit = diam / max_speed(dim, cells, h, adv[2], seg, data)
    assert O.advection_courant(om, p, adv, dt_crit * (1 - 1e-9))
    assert not O.advection_courant(om, p, adv, dt_crit * (1 + 1e-9))
    # no segments: never violated
    assert O.advection_courant(om, p, (np.full_like(seg, -1), data, adv[2]), 1e9)
    # the cut-off's irrelevant grains do not count
    mask = np.random.default_rng(32).integers(0, 1 << G, int(np.prod(cells))).astype(np.uint16)
    dt_m = diam / max_speed(dim, cells, h, adv[2], seg, data, mask)
    assert dt_m >= dt_crit
    assert O.advection_courant(om, p, adv, dt_m * (1 - 1e-9), mask=mask)
    assert not O.advection_courant(om, p, adv, dt_m * (1 + 1e-9), mask=mask)


@pytest.mark.parametrize("dim,cells,G", [(2, (7, 6), 3), (3, (4, 4, 3), 2)])
def test_preconditioner_diagonals_with_advection(dim, cells, G):
    """precondition_advection_ch / _ac (operator_sintering_generic.h:800-850):
    the block preconditioner's diagonals gain the diagonal of the advection
    terms, i.e. what J v with advection adds on the diagonal (probed with
    nodes two apart, whose supports share no cell)."""
    om, p = oracle_mesh(dim, cells), O.make_params(G, tensorial=True)
    u = random_state(dim, cells, G, seed=41)
    seg, data = advection_data(dim, cells, G, seed=42)
    adv = (seg, data, (0.0, 0.0, 0.0))
    T = O.make_time(10.0, 1.0, [-10.0])
    C, N = G + 2, u.shape[1]
    nn = [c + 1 for c in cells]
    co = np.stack([(np.arange(N) // int(np.prod(nn[:d]))) % nn[d] for d in range(dim)])
    colour = sum((co[d] % 2) << d for d in range(dim))
    diag = np.zeros((C, N))
    for comp in [0] + list(range(2, C)):
        for col in range(1 << dim):
            probe = np.zeros((C, N))
            probe[comp, colour == col] = 1.0
            d = O.jvp(om, p, T, u, probe, advection=adv) - O.jvp(om, p, T, u, probe)
            diag[comp, colour == col] = d[comp, colour == col]
    ch = O.ch_blocks(om, p, T, u, advection=adv) - O.ch_blocks(om, p, T, u)
    ac = O.ac_diagonal(om, p, T, u, advection=adv) - O.ac_diagonal(om, p, T, u)
    scale = np.abs(diag).max()
    assert scale > 1e-3
    assert np.allclose(ch[0], diag[0], atol=1e-12 * scale, rtol=0)
    assert not ch[1:].any()  # the c-mu, mu-c and mu-mu entries do not change
    assert np.allclose(ac, diag[2:], atol=1e-12 * scale, rtol=0)
