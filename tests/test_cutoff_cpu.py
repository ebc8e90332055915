"""The grain cut-off in the CPU oracle (no GPU).

SinteringOperatorData::set_component_mask (operator_sintering_data.h:149-203)
marks grain b relevant on a cell when the largest |eta_b| over the cell's
nodes exceeds the tolerance; do_vmult_range_no_template and
do_evaluate_nonlinear_residual_nt (operator_sintering_generic.h:456-537,
:1008-1081) then treat every cell with c, mu and its relevant grains only.
These tests pin the oracle's restatement: the mask rule, the all-grains mask
as the full operator, exactness where a grain is identically zero, and the
Jacobian of the cut-off residual (central differences at a fixed mask, as
tests/tangent_generic_*.cc check the full operator).
"""
import numpy as np
import pytest

from helpers import block_rel_err, grain_mask_numpy, oracle_mesh, particle_state, random_state
from oracle import oracle as O

CASES = [
    # dim, cells, G, tensorial
    (2, (13, 9), 4, True),
    (2, (13, 9), 4, False),
    (3, (7, 6, 5), 5, True),
    (3, (6, 5, 4), 3, False),
]


def ids(c):
    return f"{c[0]}d-G{c[2]}-{'tens' if c[3] else 'scal'}"


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_mask_rule(case):
    dim, cells, G, tens = case
    u = particle_state(dim, cells, G, seed=3)
    p = O.make_params(G, tensorial=tens)
    for tol in (1e-8, 1e-3, 0.2, 0.99):
        m = O.grain_mask(oracle_mesh(dim, cells), p, u, tol)
        assert np.array_equal(m, grain_mask_numpy(dim, cells, G, u, tol)), tol
    # tolerance 1: no grain anywhere (these states have eta < 1)
    assert not O.grain_mask(oracle_mesh(dim, cells), p, u, 1.0).any()


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_all_grains_mask_is_the_full_operator(case):
    dim, cells, G, tens = case
    om, p = oracle_mesh(dim, cells), O.make_params(G, tensorial=tens)
    u = random_state(dim, cells, G, seed=1)
    old = random_state(dim, cells, G, seed=2)
    src = random_state(dim, cells, G, seed=3, smooth=False) - 0.5
    full = np.full(int(np.prod(cells)), (1 << G) - 1, dtype=np.uint16)
    T = O.make_time(20.0, 1.0, [-20.0])
    assert np.array_equal(O.residual(om, p, T, u, [old], 2, mask=full), O.residual(om, p, T, u, [old], 2))
    assert np.array_equal(O.jvp(om, p, T, u, src, mask=full), O.jvp(om, p, T, u, src))
    assert np.array_equal(O.ac_diagonal(om, p, T, u, mask=full), O.ac_diagonal(om, p, T, u))
    assert np.array_equal(O.ch_blocks(om, p, T, u, mask=full), O.ch_blocks(om, p, T, u))


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_cut_off_is_exact_where_a_grain_vanishes(case):
    """A grain that is identically zero (state and direction) on the cells
    where it is cut changes nothing but its own (zero) rows: the cut-off only
    drops terms that vanish."""
    dim, cells, G, tens = case
    om, p = oracle_mesh(dim, cells), O.make_params(G, tensorial=tens)
    u = particle_state(dim, cells, G, seed=5)
    src = random_state(dim, cells, G, seed=6, smooth=False) - 0.5
    u[2 + 1] = 0.0    # grain 1 is absent everywhere
    src[2 + 1] = 0.0
    assert not (O.grain_mask(om, p, u, 0.0) & 2).any()  # the rule cuts it everywhere
    mask = np.full(int(np.prod(cells)), ((1 << G) - 1) & ~2, dtype=np.uint16)  # and nothing else
    T = O.make_time(20.0, 1.0, [-20.0])
    # equal up to rounding (the per-grain sums run over fewer terms, which the
    # compiled oracle may group differently)
    kw = dict(rtol=1e-13, atol=1e-14)
    np.testing.assert_allclose(O.jvp(om, p, T, u, src, mask=mask)[[0, 1, 3]], O.jvp(om, p, T, u, src)[[0, 1, 3]],
                               **kw)
    np.testing.assert_allclose(O.residual(om, p, T, u, [u], 2, mask=mask)[[0, 1]],
                               O.residual(om, p, T, u, [u], 2)[[0, 1]], **kw)
    # the cut grain's rows are empty
    assert not O.jvp(om, p, T, u, src, mask=mask)[3].any()
    assert not O.residual(om, p, T, u, [u], 2, mask=mask)[3].any()


def test_absent_grain_rows_receive_nothing():
    dim, cells, G = 3, (6, 5, 4), 4
    om, p = oracle_mesh(dim, cells), O.make_params(G)
    u = particle_state(dim, cells, G, seed=7)
    src = random_state(dim, cells, G, seed=8, smooth=False) - 0.5
    mask = np.full(int(np.prod(cells)), 0b1011, dtype=np.uint16)  # grain 2 nowhere
    T = O.make_time(20.0, 1.0, [-20.0])
    j = O.jvp(om, p, T, u, src, mask=mask)
    r = O.residual(om, p, T, u, [u], 2, mask=mask)
    d = O.ac_diagonal(om, p, T, u, mask=mask)
    assert not j[4].any() and not r[4].any() and not d[2].any()
    assert np.all(O.inverse_diagonal(d)[2] == 1.0)  # guarded inverse of the empty diagonal
    assert j[5].any() and r[5].any()


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_cut_off_jacobian_is_the_derivative_of_the_cut_off_residual(case):
    dim, cells, G, tens = case
    om, p = oracle_mesh(dim, cells), O.make_params(G, tensorial=tens)
    u = particle_state(dim, cells, G, seed=9)
    v = random_state(dim, cells, G, seed=10, smooth=False) - 0.5
    mask = O.grain_mask(om, p, u, 1e-3)
    assert 0 < np.count_nonzero(mask) and np.count_nonzero(mask != (1 << G) - 1) > 0
    T = O.make_time(20.0, 1.0, [-20.0])
    eps = 1e-6
    fd = (O.residual(om, p, T, u + eps * v, [u], 2, mask=mask) -
          O.residual(om, p, T, u - eps * v, [u], 2, mask=mask)) / (2 * eps)
    jv = O.jvp(om, p, T, u, v, mask=mask)
    # hpsint's tensorial tangent leaves out the derivative of the grain-boundary
    # projectors by grad eta (mobility.h:808-916), so its c row is not the exact
    # derivative at grain boundaries -- with or without the cut-off; the other
    # rows, and every row with scalar mobility, are
    rows = slice(1, None) if tens else slice(None)
    assert block_rel_err(jv[rows], fd[rows]) <= 1e-6
