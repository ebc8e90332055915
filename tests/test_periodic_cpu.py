"""Periodic constraints in the CPU oracle (no GPU).

hpsint makes a mesh periodic with DoFTools::make_periodicity_constraints
(sintering/driver.h:629-643): the nodes at the upper face of a periodic
direction become slaves of the lower face's, and the constrained operators
(OperatorBase::vmult, operator_base.h:294-353) read masters for slaves, add
the slave rows to the master rows and give the slave rows the identity
(J v) or zero (residual).  The oracle restates that; these tests pin it to a
genuinely periodic computation: the same state tiled three times along each
periodic direction, where the middle copy's rows see their neighbours
across the period.
"""
import itertools

import numpy as np
import pytest

from oracle import oracle as O


def periodic_state(dim, cells, G, dirs, seed):
    """Random smooth-ish state with slaves equal to masters, and its values
    on the unique nodes (shape C x unique grid, x fastest)."""
    rng = np.random.default_rng(seed)
    un = [cells[d] if d in dirs else cells[d] + 1 for d in range(dim)]
    C = G + 2
    uniq = rng.uniform(0.05, 0.95, size=(C,) + tuple(reversed(un)))
    nn = [cells[d] + 1 for d in range(dim)]
    idx = [np.arange(nn[d]) % un[d] for d in range(dim)]
    full = uniq[(slice(None),) + tuple(np.ix_(*[idx[d] for d in reversed(range(dim))]))]
    return full.reshape(C, -1), uniq


def tiled(dim, cells, dirs, uniq, copies=3):
    """State on the mesh tiled `copies` times along the periodic directions."""
    un = [cells[d] if d in dirs else cells[d] + 1 for d in range(dim)]
    big = [copies * cells[d] if d in dirs else cells[d] for d in range(dim)]
    idx = [np.arange(big[d] + 1) % un[d] for d in range(dim)]
    full = uniq[(slice(None),) + tuple(np.ix_(*[idx[d] for d in reversed(range(dim))]))]
    return big, full.reshape(uniq.shape[0], -1)


def middle_rows(dim, cells, dirs, big):
    """Indices, in the tiled mesh, of the original mesh's non-slave nodes
    (taken from the middle copy), in the original node order."""
    nn = [cells[d] + 1 for d in range(dim)]
    bn = [big[d] + 1 for d in range(dim)]
    rows, orig = [], []
    for co in itertools.product(*[range(nn[d]) for d in reversed(range(dim))]):
        co = tuple(reversed(co))
        if any(d in dirs and co[d] == cells[d] for d in range(dim)):
            continue
        bco = [co[d] + (cells[d] if d in dirs else 0) for d in range(dim)]
        rows.append(sum(bco[d] * int(np.prod(bn[:d])) for d in range(dim)))
        orig.append(sum(co[d] * int(np.prod(nn[:d])) for d in range(dim)))
    return np.array(rows), np.array(orig)


CASES = [(2, (6, 5), 3, (0,)), (2, (6, 5), 3, (0, 1)), (3, (4, 3, 3), 2, (0,)), (3, (4, 3, 3), 3, (0, 2)),
         (3, (3, 3, 3), 2, (0, 1, 2))]


@pytest.mark.parametrize("dim,cells,G,dirs", CASES)
@pytest.mark.parametrize("tens", [True, False])
def test_constrained_operator_is_the_periodic_operator(dim, cells, G, dirs, tens):
    p = O.make_params(G, tensorial=tens)
    om = O.make_mesh(dim, list(cells) + [0] * (3 - dim))
    u, uu = periodic_state(dim, cells, G, dirs, seed=1)
    old, uo = periodic_state(dim, cells, G, dirs, seed=2)
    src, us = periodic_state(dim, cells, G, dirs, seed=3)
    T = O.make_time(10.0, 1.0, [-10.0])
    big, ub = tiled(dim, cells, dirs, uu)
    _, ob = tiled(dim, cells, dirs, uo)
    _, sb = tiled(dim, cells, dirs, us)
    bm = O.make_mesh(dim, list(big) + [0] * (3 - dim))
    rows, orig = middle_rows(dim, cells, dirs, big)
    jv = O.periodic_jvp(om, p, T, u, src, dirs)
    assert np.allclose(jv[:, orig], O.jvp(bm, p, T, ub, sb)[:, rows], rtol=1e-12, atol=1e-12)
    r = O.periodic_residual(om, p, T, u, [old], 2, dirs)
    assert np.allclose(r[:, orig], O.residual(bm, p, T, ub, [ob], 2)[:, rows], rtol=1e-12, atol=1e-12)
    sl, ma = O.periodic_pairs(om, dirs)
    assert np.array_equal(jv[:, sl], src[:, sl]) and not r[:, sl].any()


def test_slaves_are_ignored_on_input():
    """The constrained operators read masters wherever a slave is: garbage in
    the slave entries of the input changes nothing but the identity rows."""
    dim, cells, G, dirs = 2, (6, 5), 2, (0, 1)
    p, om = O.make_params(G), O.make_mesh(2, [6, 5, 0])
    u, _ = periodic_state(dim, cells, G, dirs, seed=4)
    src, _ = periodic_state(dim, cells, G, dirs, seed=5)
    sl, ma = O.periodic_pairs(om, dirs)
    src2 = src.copy()
    src2[:, sl] = 7.0
    T = O.make_time(10.0, 1.0, [-10.0])
    a, b = O.periodic_jvp(om, p, T, u, src, dirs), O.periodic_jvp(om, p, T, u, src2, dirs)
    keep = np.setdiff1d(np.arange(u.shape[1]), sl)
    assert np.array_equal(a[:, keep], b[:, keep]) and np.all(b[:, sl] == 7.0)


def test_particle_groups():
    """PeriodicityGraph::build_groups (periodicity_graph.h:57-80): particles
    connected through periodicity pairs form one group; particles outside
    the graph have none."""
    from hpsint_b200.grain_tracker import particle_groups
    ids, n = particle_groups(6, [(0, 4), (4, 5), (2, 2)])
    assert n == 2 and ids == [0, -1, 1, -1, 0, 0]
    assert particle_groups(3, []) == ([-1, -1, -1], 0)
    # order of the pairs does not matter
    a = particle_groups(8, [(6, 7), (1, 3), (3, 6), (2, 5)])
    b = particle_groups(8, [(2, 5), (3, 6), (6, 7), (1, 3)])
    assert a == b == ([-1, 0, 1, 0, -1, 1, 0, 0], 2)


def test_segment_periodicity_pairs():
    """Pairs of particles owning cells that face each other across a periodic
    boundary (tracker.h:1290-1336), in increasing order, without repeats."""
    mesh = O.make_mesh(2, [4, 3, 0])
    ids = np.array([[0, -1, -1, 1],
                    [0, -1, 2, 2],
                    [-1, -1, -1, 3]]).ravel()  # rows = y, x fastest
    assert O.segment_periodicity(mesh, ids, (0,)) == [(0, 1), (0, 2)]
    assert O.segment_periodicity(mesh, ids, (1,)) == [(1, 3)]
    assert O.segment_periodicity(mesh, ids, (0, 1)) == [(0, 1), (0, 2), (1, 3)]


@pytest.mark.parametrize("dim,cells,G,dirs", [(2, (6, 5), 3, (0, 1)), (3, (4, 3, 3), 2, (0, 2))])
def test_periodic_operator_with_translation(dim, cells, G, dirs):
    """Periodic constraints and advection together: with translations only
    (the velocity field is then periodic) the constrained operator with
    advection equals the tiled operator with the same velocities."""
    p = O.make_params(G, tensorial=True)
    om = O.make_mesh(dim, list(cells) + [0] * (3 - dim))
    u, uu = periodic_state(dim, cells, G, dirs, seed=11)
    src, us = periodic_state(dim, cells, G, dirs, seed=12)
    T = O.make_time(10.0, 1.0, [-10.0])
    big, ub = tiled(dim, cells, dirs, uu)
    _, sb = tiled(dim, cells, dirs, us)
    bm = O.make_mesh(dim, list(big) + [0] * (3 - dim))
    rng = np.random.default_rng(13)
    data = np.zeros((G, 9))
    data[:, :dim] = rng.normal(size=(G, dim))
    seg = np.repeat(np.arange(G, dtype=np.int32)[:, None], int(np.prod(cells)), axis=1)
    seg_b = np.repeat(np.arange(G, dtype=np.int32)[:, None], int(np.prod(big)), axis=1)
    rows, orig = middle_rows(dim, cells, dirs, big)
    jv = O.periodic_jvp(om, p, T, u, src, dirs, advection=(seg, data, (0, 0, 0)))
    ref = O.jvp(bm, p, T, ub, sb, advection=(seg_b, data, (0, 0, 0)))
    assert np.allclose(jv[:, orig], ref[:, rows], rtol=1e-12, atol=1e-12)
    r = O.periodic_residual(om, p, T, u, [u], 2, dirs, advection=(seg, data, (0, 0, 0)))
    rb = O.residual(bm, p, T, ub, [ub], 2, advection=(seg_b, data, (0, 0, 0)))
    assert np.allclose(r[:, orig], rb[:, rows], rtol=1e-12, atol=1e-12)
    # the translation changed the operator
    assert not np.allclose(jv, O.periodic_jvp(om, p, T, u, src, dirs), rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("dim,cells,G,dirs", [(2, (6, 5), 3, (0, 1)), (3, (4, 3, 3), 2, (0, 2))])
def test_condensed_preconditioner_diagonals_are_periodic(dim, cells, G, dirs):
    """The preconditioner's diagonals condensed over the periodic pairs equal
    the diagonals of the tiled (genuinely periodic) operator."""
    p = O.make_params(G, tensorial=True)
    om = O.make_mesh(dim, list(cells) + [0] * (3 - dim))
    u, uu = periodic_state(dim, cells, G, dirs, seed=21)
    T = O.make_time(10.0, 1.0, [-10.0])
    big, ub = tiled(dim, cells, dirs, uu)
    bm = O.make_mesh(dim, list(big) + [0] * (3 - dim))
    rows, orig = middle_rows(dim, cells, dirs, big)
    raw = np.concatenate([O.ch_blocks(om, p, T, u), O.ac_diagonal(om, p, T, u)])
    ours = O.periodic_condense(om, raw, None, dirs, 2)
    ref = np.concatenate([O.ch_blocks(bm, p, T, ub), O.ac_diagonal(bm, p, T, ub)])
    assert np.allclose(ours[:, orig], ref[:, rows], rtol=1e-12, atol=1e-12)
