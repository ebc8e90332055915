"""Size-independent properties of the oracle's operator, on which the GPU
parity at full sizes rests: J(u) v is linear in v, and the residual, J v, the
Allen-Cahn diagonal and the Cahn-Hilliard blocks are equivariant under a
relabelling of the grains.  The free energy and the mobility are symmetric in
the order parameters (sintering/free_energy.h, sintering/mobility.h of
hpsint), so permuting the eta components of the state permutes the eta rows
of every result and leaves the c and mu rows unchanged, up to the rounding of
the grain sums taken in another order."""
import numpy as np
import pytest

from helpers import block_rel_err, oracle_mesh, random_state
from oracle import oracle as O

CASES = [(2, (7, 6), 4, False), (2, (7, 6), 4, True), (3, (4, 3, 3), 3, False), (3, (4, 3, 3), 3, True)]


def _case(dim, cells, G, tensorial, seed=3):
    mesh = oracle_mesh(dim, cells)
    prm = O.make_params(G, tensorial=tensorial)
    tm = O.make_time(10.0, 1.0, [-10.0])
    u = random_state(dim, cells, G, seed)
    u_old = random_state(dim, cells, G, seed + 100)
    return mesh, prm, tm, u, u_old


def _permute(x, perm):
    """Relabel the grains of a (G + 2, N) block vector: new grain k = old perm[k]."""
    return np.concatenate([x[:2], x[2:][perm]])


@pytest.mark.parametrize("dim,cells,G,tensorial", CASES)
def test_jvp_is_linear_in_v(dim, cells, G, tensorial):
    mesh, prm, tm, u, _ = _case(dim, cells, G, tensorial)
    rng = np.random.default_rng(11)
    v1, v2 = rng.standard_normal(u.shape), rng.standard_normal(u.shape)
    a, b = 0.75, -1.5
    lhs = O.jvp(mesh, prm, tm, u, a * v1 + b * v2)
    rhs = a * O.jvp(mesh, prm, tm, u, v1) + b * O.jvp(mesh, prm, tm, u, v2)
    assert block_rel_err(lhs, rhs) < 1e-12


@pytest.mark.parametrize("dim,cells,G,tensorial", CASES)
def test_operator_is_equivariant_under_grain_relabelling(dim, cells, G, tensorial):
    mesh, prm, tm, u, u_old = _case(dim, cells, G, tensorial)
    v = np.random.default_rng(5).standard_normal(u.shape)
    perm = np.roll(np.arange(G), 1)[::-1].copy()
    assert not np.array_equal(perm, np.arange(G))
    up, uop, vp = _permute(u, perm), _permute(u_old, perm), _permute(v, perm)

    r, rp = O.residual(mesh, prm, tm, u, [u_old], 2), O.residual(mesh, prm, tm, up, [uop], 2)
    assert block_rel_err(rp, _permute(r, perm)) < 1e-12
    j, jp = O.jvp(mesh, prm, tm, u, v), O.jvp(mesh, prm, tm, up, vp)
    assert block_rel_err(jp, _permute(j, perm)) < 1e-12
    d, dp = O.ac_diagonal(mesh, prm, tm, u), O.ac_diagonal(mesh, prm, tm, up)
    assert block_rel_err(dp, d[perm]) < 1e-12
    ch, chp = O.ch_blocks(mesh, prm, tm, u), O.ch_blocks(mesh, prm, tm, up)
    assert block_rel_err(chp, ch) < 1e-12


@pytest.mark.parametrize("tensorial", [False, True])
def test_relabelling_is_not_trivially_satisfied(tensorial):
    """The check above has teeth: swapping the eta rows of the result without
    relabelling the state breaks it (the grains' fields differ)."""
    mesh, prm, tm, u, u_old = _case(2, (7, 6), 4, tensorial)
    perm = np.array([1, 0, 2, 3])
    r = O.residual(mesh, prm, tm, u, [u_old], 2)
    assert block_rel_err(_permute(r, perm), r) > 1e-3


@pytest.mark.parametrize("dim,cells,G,tensorial", CASES[::2])
def test_residual_history_enters_linearly(dim, cells, G, tensorial):
    """The history h enters the residual only through the time-derivative
    mass term w_1 (phi_i, h) of the c and eta rows (BDF1 here): R(u, [h]) is
    affine in h and its mu row does not depend on h."""
    mesh, prm, tm, u, u_old = _case(dim, cells, G, tensorial)
    rng = np.random.default_rng(17)
    h1, h2 = u_old, u_old + 0.05 * rng.standard_normal(u.shape)
    a, b = 0.4, 0.6
    R = lambda h: O.residual(mesh, prm, tm, u, [h], 2)
    r0 = R(np.zeros_like(u))
    d1, d2 = R(h1) - r0, R(h2) - r0
    d12 = R(a * h1 + b * h2) - r0
    assert block_rel_err(d12[[0] + list(range(2, G + 2))], (a * d1 + b * d2)[[0] + list(range(2, G + 2))]) < 1e-10
    assert np.max(np.abs(d1[1])) <= 1e-14 * max(1.0, np.max(np.abs(r0[1])))
    assert np.max(np.abs(d1[0])) > 1e-3  # the history does act on the c row
