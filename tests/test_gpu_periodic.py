"""Periodic constraints on the GPU against the CPU oracle.

The oracle's constrained operators are pinned to the genuinely periodic
(tiled) operator on the CPU (tests/test_periodic_cpu.py); here the device
residual, J v (FP64, FP32), preconditioner diagonals and Newton solve with
periodic directions match them: 1e-12 per-block relative in FP64, 2e-5 in
FP32, the Newton step to 1e-7 against a CPU Newton on the oracle.
"""
import numpy as np
import pytest

from helpers import block_rel_err, oracle_mesh, particle_state, random_state
from oracle import oracle as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def make_op(dim, cells, G, tensorial, dirs):
    import hpsint_b200 as hb
    op = hb.SinteringOperatorGeneric(hb.Mesh(dim, tuple(cells) + (1,) * (3 - len(cells))),
                                     hb.Params(G, tensorial=tensorial))
    op.set_periodicity(dirs)
    return op, O.make_params(G, tensorial=tensorial), oracle_mesh(dim, cells)


CASES = [
    # dim, cells, G, tensorial, periodic directions
    (2, (37, 21), 4, True, (0,)),
    (2, (37, 21), 3, False, (0, 1)),
    (2, (16, 16), 9, True, (0, 1)),
    (3, (13, 11, 9), 5, True, (0, 2)),
    (3, (9, 8, 7), 3, False, (0, 1, 2)),
    (3, (8, 12, 5), 9, True, (1,)),
]


def ids(c):
    return f"{c[0]}d-G{c[2]}-{'tens' if c[3] else 'scal'}-p{''.join(map(str, c[4]))}"


def distributed(om, u, dirs):
    return O.periodic_resolve(om, u, dirs)


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_residual_and_jacobian_match_oracle(case):
    dim, cells, G, tens, dirs = case
    op, p, om = make_op(dim, cells, G, tens, dirs)
    u = distributed(om, particle_state(dim, cells, G, seed=81), dirs)
    old = distributed(om, particle_state(dim, cells, G, seed=81, width=1.2), dirs)
    src = random_state(dim, cells, G, seed=82, smooth=False) - 0.5  # slaves not distributed: must be ignored
    op.set_time_weights(20.0, [-20.0], 1.0)
    T = O.make_time(20.0, 1.0, [-20.0])
    ud = op.to_device(u)
    r = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(r, ud, 2, [op.to_device(old)])
    op.fill_quadrature_point_values(ud)
    j = op.initialize_dof_vector()
    op.vmult(j, op.to_device(src))
    j32 = op.initialize_dof_vector(torch.float32)
    op.vmult(j32, op.to_device(src, torch.float32))
    torch.cuda.synchronize()
    r_ref = O.periodic_residual(om, p, T, u, [old], 2, dirs)
    j_ref = O.periodic_jvp(om, p, T, u, src, dirs)
    assert block_rel_err(op.to_host(r), r_ref) <= 1e-12
    assert block_rel_err(op.to_host(j), j_ref) <= 1e-12
    src32 = src.astype(np.float32).astype(np.float64)
    u32 = u.astype(np.float32).astype(np.float64)
    assert block_rel_err(op.to_host(j32), O.periodic_jvp(om, p, T, u32, src32, dirs)) <= 2e-5
    # periodicity changed the operator
    assert block_rel_err(j_ref, O.jvp(om, p, T, u, src)) > 1e-6


@pytest.mark.parametrize("case", CASES[:4], ids=[ids(c) for c in CASES[:4]])
def test_preconditioner_diagonals_match_oracle(case):
    import hpsint_b200 as hb
    dim, cells, G, tens, dirs = case
    op, p, om = make_op(dim, cells, G, tens, dirs)
    u = distributed(om, particle_state(dim, cells, G, seed=83), dirs)
    op.set_time_weights(40.0, [-40.0], 1.0)
    op.fill_quadrature_point_values(op.to_device(u))
    pc = hb.BlockPreconditioner2(op)
    pc.do_update()
    T = O.make_time(40.0, 1.0, [-40.0])
    raw = np.concatenate([O.ch_blocks(om, p, T, u), O.ac_diagonal(om, p, T, u)])
    ref = O.periodic_condense(om, raw, None, dirs, 2)
    N = op.N
    assert block_rel_err(pc.ch_blocks()[:, :N].cpu().numpy(), ref[:4]) <= 1e-12
    assert block_rel_err(pc.inverse_diagonal()[:, :N].cpu().numpy(), O.inverse_diagonal(ref[4:])) <= 1e-12


def test_periodic_under_the_cut_off():
    dim, cells, G, dirs = 3, (14, 9, 10), 6, (0, 1)
    op, p, om = make_op(dim, cells, G, True, dirs)
    u = distributed(om, particle_state(dim, cells, G, seed=84), dirs)
    src = random_state(dim, cells, G, seed=85, smooth=False) - 0.5
    ud = op.to_device(u)
    op.set_component_mask(ud, 1e-3)
    mask = O.grain_mask(om, p, u, 1e-3)
    op.set_time_weights(20.0, [-20.0], 1.0)
    op.fill_quadrature_point_values(ud)
    j = op.initialize_dof_vector()
    op.vmult(j, op.to_device(src))
    torch.cuda.synchronize()
    T = O.make_time(20.0, 1.0, [-20.0])
    assert block_rel_err(op.to_host(j), O.periodic_jvp(om, p, T, u, src, dirs, mask=mask)) <= 1e-12


def _wrapped_particles(cells, R=6.0):
    """Two particles, the first centred on the x = 0 boundary (half of it on
    each side of the periodic direction)."""
    from hpsint_b200 import packings as P
    nx, ny = cells
    c = np.array([[0.0, ny / 2], [2 * R - 1.0, ny / 2], [float(nx), ny / 2]])
    # the image of particle 0 at x = nx carries the same order parameter
    return P.initial_state(2, cells, (1.0, 1.0), (0.0, 0.0), c, np.array([R, R, R]), np.array([0, 1, 0]),
                           width=2.0, noise=1e-3, seed=5)


def _cpu_newton(om, P, T, u_old, dirs, tol_rel=1e-12, max_it=30):
    from scipy.sparse.linalg import LinearOperator, gmres
    u = u_old.copy()
    C, N = u.shape
    r0 = None
    for _ in range(max_it):
        r = O.periodic_residual(om, P, T, u, [u_old], 2, dirs)
        nr = np.linalg.norm(r)
        r0 = nr if r0 is None else r0
        if nr <= tol_rel * r0 or nr < 1e-14:
            return O.periodic_resolve(om, u, dirs)
        lin = u.copy()
        J = LinearOperator((C * N, C * N),
                           matvec=lambda v: O.periodic_jvp(om, P, T, lin, v.reshape(C, N), dirs).ravel())
        du, info = gmres(J, -r.ravel(), rtol=1e-13, atol=0.0, restart=300, maxiter=50)
        u = u + du.reshape(C, N)
    raise RuntimeError("CPU Newton did not converge")


@pytest.mark.parametrize("prec", [64, 32])
def test_newton_with_periodic_directions(prec):
    import hpsint_b200 as hb
    cells, G, dt, dirs = (40, 20), 2, 1e-2, (0,)
    om = oracle_mesh(2, cells)
    u_old = O.periodic_resolve(om, _wrapped_particles(cells), dirs)
    P = O.make_params(G, tensorial=True)
    T = O.make_time(1.0 / dt, 1.0, [-1.0 / dt])
    ref = _cpu_newton(om, P, T, u_old, dirs)
    op, _, _ = make_op(2, cells, G, True, dirs)
    op.set_time_weights(1.0 / dt, [-1.0 / dt], 1.0)
    old = op.to_device(u_old)
    u = old.clone()
    st = hb.DampedNewtonSolver(op, hb.NonLinearData(nl_rel_tol=1e-10, nl_abs_tol=1e-16, l_rel_tol=1e-4,
                                                    nl_max_iter=20, inner_precision=prec)).solve(u, [old])
    torch.cuda.synchronize()
    assert st.status == 0
    uh = op.to_host(u)
    assert np.max(np.abs(uh - ref)) < (1e-7 if prec == 64 else 1e-6)
    sl, ma = O.periodic_pairs(om, dirs)
    assert np.array_equal(uh[:, sl], uh[:, ma])  # distributed at the end of the solve
    # the periodic step differs from the one on the box
    assert np.max(np.abs(ref - u_old)) > 1e-4


def test_distribute_constraints():
    dim, cells, G, dirs = 3, (6, 5, 4), 2, (0, 1, 2)
    op, p, om = make_op(dim, cells, G, False, dirs)
    u = random_state(dim, cells, G, seed=86, smooth=False)
    ud = op.to_device(u)
    op.distribute_constraints(ud)
    torch.cuda.synchronize()
    assert np.array_equal(op.to_host(ud), O.periodic_resolve(om, u, dirs))


def test_advection_forces_read_periodic_masters():
    """The force evaluation reads the periodic masters as the operator does,
    so stale slave entries of an iterate do not enter the velocities."""
    from helpers import advection_data
    dim, cells, G, dirs = 2, (37, 21), 3, (0, 1)
    op, p, om = make_op(dim, cells, G, True, dirs)
    u = distributed(om, particle_state(dim, cells, G, seed=87), dirs)
    sl, ma = O.periodic_pairs(om, dirs)
    stale = u.copy()
    stale[:, sl] += 0.3
    seg, data = advection_data(dim, cells, G, seed=88)
    centers = np.ascontiguousarray(data[:, 6:9])
    op.set_advection_mechanism(torch.from_numpy(seg).cuda(), torch.from_numpy(centers).cuda(), k=2.5, cgb=0.0,
                               ceq=0.9, smoothening=0.0, mt=1.0, mr=1.0)
    vft = op.advection_forces(op.to_device(stale)).cpu().numpy()
    ref = O.advection_forces(om, p, u, seg, centers, (0.0, 0.0, 0.0), 2.5, 0.0, 0.9, 0.0)
    scale = np.abs(ref).max(axis=0, keepdims=True)
    assert np.all(np.abs(vft - ref) <= 1e-12 * scale + 1e-300)


@pytest.mark.parametrize("prec", [64, 32])
def test_cut_off_across_the_periodic_boundary(prec):
    """Grain cut-off on a periodic mesh with a particle cut by the boundary:
    the nodes there see the cells of both sides, so skipping GMRES's dead
    chunks changes nothing (bitwise) and the step matches the one without
    the cut-off to the cut-off's tolerance."""
    import hpsint_b200 as hb
    cells, G, dt, dirs = (40, 20), 2, 1e-2, (0, 1)
    om = oracle_mesh(2, cells)
    u_old = O.periodic_resolve(om, _wrapped_particles(cells), dirs)
    out = {}
    for tol, skip in ((0.0, True), (1e-5, True), (1e-5, False)):
        op, _, _ = make_op(2, cells, G, True, dirs)
        op.set_time_weights(1.0 / dt, [-1.0 / dt], 1.0)
        old = op.to_device(u_old)
        op.set_component_mask(old, tol)
        if tol:
            op.set_cut_off_skip_zero_chunks(skip)
        u = old.clone()
        st = hb.DampedNewtonSolver(op, hb.NonLinearData(nl_rel_tol=1e-9, nl_abs_tol=1e-16,
                                                        inner_precision=prec)).solve(u, [old])
        torch.cuda.synchronize()
        assert st.status == 0
        out[(tol, skip)] = u
    assert torch.equal(out[(1e-5, True)], out[(1e-5, False)])
    assert (out[(1e-5, True)] - out[(0.0, True)]).abs().max().item() < 1e-3
