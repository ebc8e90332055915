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

from helpers import advection_data, oracle_mesh, random_state
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
