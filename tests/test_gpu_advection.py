"""Advection (grain rigid-body motion) on the GPU against the CPU oracle.

The residual and Jacobian products with given segment velocities meet the
full operator's tolerances (FP64 1e-12 per-block relative, FP32 2e-5 against
the oracle at FP32-rounded inputs), alone and under the grain cut-off;
switching advection off gives back the operator bit for bit; the device
Newton solve with advection converges to the oracle's step; graph-replayed
solves read the current velocities.
"""
import numpy as np
import pytest

from helpers import advection_data, block_rel_err, max_speed, oracle_mesh, particle_state, random_state
from oracle import oracle as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

ORIGIN = (1.5, -2.0, 0.25)
H = (0.9, 1.1, 1.0)


def make_op(dim, cells, G, tensorial, h=H, origin=ORIGIN):
    import hpsint_b200 as hb
    mesh = hb.Mesh(dim, tuple(cells) + (1,) * (3 - len(cells)), tuple(h), tuple(origin))
    om = O.make_mesh(dim, list(cells) + [0] * (3 - dim), h)
    return hb.SinteringOperatorGeneric(mesh, hb.Params(G, tensorial=tensorial)), O.make_params(G, tensorial=tensorial), om


def set_adv(op, seg, data):
    op.set_advection(torch.from_numpy(seg).cuda().contiguous(), torch.from_numpy(data).cuda().contiguous())


CASES = [
    # dim, cells, G, tensorial
    (2, (37, 21), 3, True),
    (2, (37, 21), 4, False),
    (2, (30, 26), 9, True),
    (3, (13, 11, 9), 5, True),
    (3, (13, 11, 9), 3, False),
    (3, (11, 9, 10), 9, True),
]


def ids(c):
    return f"{c[0]}d-G{c[2]}-{'tens' if c[3] else 'scal'}"


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_residual_and_jacobian_match_oracle(case):
    dim, cells, G, tens = case
    op, p, om = make_op(dim, cells, G, tens)
    u = particle_state(dim, cells, G, seed=41)
    old = particle_state(dim, cells, G, seed=41, width=1.2)
    src = random_state(dim, cells, G, seed=42, smooth=False) - 0.5
    seg, data = advection_data(dim, cells, G, seed=43, scale=5.0)
    set_adv(op, seg, data)
    adv = (seg, data, ORIGIN)
    op.set_time_weights(20.0, [-20.0], 1.0)
    T = O.make_time(20.0, 1.0, [-20.0])
    ud = op.to_device(u)
    r = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(r, ud, 2, [op.to_device(old)])
    op.fill_quadrature_point_values(ud)
    j = op.initialize_dof_vector()
    op.vmult(j, op.to_device(src))
    torch.cuda.synchronize()
    r_ref = O.residual(om, p, T, u, [old], 2, advection=adv)
    j_ref = O.jvp(om, p, T, u, src, advection=adv)
    assert block_rel_err(op.to_host(r), r_ref) <= 1e-12
    assert block_rel_err(op.to_host(j), j_ref) <= 1e-12
    # advection changed the result
    assert block_rel_err(j_ref, O.jvp(om, p, T, u, src)) > 1e-6
    assert block_rel_err(r_ref, O.residual(om, p, T, u, [old], 2)) > 1e-6
    # residual without the time derivative (with_time_derivative 0) too
    r0 = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(r0, ud, 0)
    torch.cuda.synchronize()
    assert block_rel_err(op.to_host(r0), O.residual(om, p, T, u, [], 0, advection=adv)) <= 1e-12


@pytest.mark.parametrize("case", CASES[:4], ids=[ids(c) for c in CASES[:4]])
def test_jacobian_f32_close_to_oracle(case):
    dim, cells, G, tens = case
    op, p, om = make_op(dim, cells, G, tens)
    u = particle_state(dim, cells, G, seed=44).astype(np.float32).astype(np.float64)
    src = (random_state(dim, cells, G, seed=45, smooth=False) - 0.5).astype(np.float32).astype(np.float64)
    seg, data = advection_data(dim, cells, G, seed=46, scale=5.0)
    set_adv(op, seg, data)
    op.set_time_weights(20.0, [-20.0], 1.0)
    op.fill_quadrature_point_values(op.to_device(u))
    j = op.initialize_dof_vector(torch.float32)
    op.vmult(j, op.to_device(src, torch.float32))
    torch.cuda.synchronize()
    j_ref = O.jvp(om, p, O.make_time(20.0, 1.0, [-20.0]), u, src, advection=(seg, data, ORIGIN))
    assert block_rel_err(op.to_host(j), j_ref) <= 2e-5


@pytest.mark.parametrize("case", [CASES[0], CASES[3], CASES[5]], ids=[ids(c) for c in (CASES[0], CASES[3], CASES[5])])
def test_advection_under_the_cut_off(case):
    dim, cells, G, tens = case
    op, p, om = make_op(dim, cells, G, tens)
    u = particle_state(dim, cells, G, seed=47)
    src = random_state(dim, cells, G, seed=48, smooth=False) - 0.5
    seg, data = advection_data(dim, cells, G, seed=49, scale=5.0)
    ud = op.to_device(u)
    op.set_component_mask(ud, 1e-3)
    mask = O.grain_mask(om, p, u, 1e-3)
    set_adv(op, seg, data)
    adv = (seg, data, ORIGIN)
    op.set_time_weights(20.0, [-20.0], 1.0)
    T = O.make_time(20.0, 1.0, [-20.0])
    r = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(r, ud, 2, [ud])
    op.fill_quadrature_point_values(ud)
    j = op.initialize_dof_vector()
    op.vmult(j, op.to_device(src))
    torch.cuda.synchronize()
    assert block_rel_err(op.to_host(r), O.residual(om, p, T, u, [u], 2, mask=mask, advection=adv)) <= 1e-12
    assert block_rel_err(op.to_host(j), O.jvp(om, p, T, u, src, mask=mask, advection=adv)) <= 1e-12


def test_switching_advection_off_is_the_plain_operator():
    dim, cells, G, tens = 3, (13, 11, 9), 4, True
    op, p, om = make_op(dim, cells, G, tens)
    u = particle_state(dim, cells, G, seed=50)
    src = random_state(dim, cells, G, seed=51, smooth=False) - 0.5
    ud, sd = op.to_device(u), op.to_device(src)
    op.set_time_weights(20.0, [-20.0], 1.0)
    op.fill_quadrature_point_values(ud)
    j0 = op.initialize_dof_vector()
    op.vmult(j0, sd)
    seg, data = advection_data(dim, cells, G, seed=52)
    set_adv(op, seg, data)
    j1 = op.initialize_dof_vector()
    op.vmult(j1, sd)
    op.set_advection(None, None)
    j2 = op.initialize_dof_vector()
    op.vmult(j2, sd)
    # no segment anywhere: the advection kernels add nothing
    set_adv(op, np.full_like(seg, -1), data)
    j3 = op.initialize_dof_vector()
    op.vmult(j3, sd)
    torch.cuda.synchronize()
    assert torch.equal(j0, j2)
    assert not torch.equal(j0, j1)
    # the advection kernels are other compiled functions: the same terms to rounding
    assert (j3 - j0).abs().max() <= 1e-14 * j0.abs().max()


def test_invalid_segment_ids_are_rejected():
    import hpsint_b200 as hb
    dim, cells, G = 2, (10, 8), 2
    op, p, om = make_op(dim, cells, G, False)
    seg, data = advection_data(dim, cells, G, seed=53)
    bad = seg.copy()
    bad[1, 17] = data.shape[0]  # one past the last segment
    with pytest.raises(hb.SintError):
        set_adv(op, bad, data)
    bad[1, 17] = -2
    with pytest.raises(hb.SintError):
        set_adv(op, bad, data)
    set_adv(op, seg, data)  # a valid table is accepted afterwards


def _two_particles(cells, R=6.0):
    from hpsint_b200 import packings as P
    nx, ny = cells
    c = np.array([[nx / 2 - R + 0.5, ny / 2], [nx / 2 + R - 0.5, ny / 2]])
    return P.initial_state(2, cells, (1.0, 1.0), (0.0, 0.0), c, np.array([R, R]), np.array([0, 1]), width=2.0,
                           noise=1e-3, seed=3)


def _two_particle_advection(cells, R=6.0, vx=2.0, w=0.3):
    """Grain 0 translates towards grain 1, grain 1 rotates about its center;
    each grain's segment covers the cells of its half of the mesh."""
    nx, ny = cells
    n_cells = nx * ny
    seg = np.full((2, n_cells), -1, dtype=np.int32)
    ci = np.arange(n_cells) % nx
    seg[0, ci < nx // 2] = 0
    seg[1, ci >= nx // 2] = 1
    data = np.zeros((2, 9))
    data[0, 0] = vx
    data[0, 6:8] = (nx / 2 - R + 0.5, ny / 2)
    data[1, 5] = w
    data[1, 6:8] = (nx / 2 + R - 0.5, ny / 2)
    return seg, data


def _cpu_newton(mesh, P, T, u_old, adv, tol_rel=1e-12, max_it=30):
    from scipy.sparse.linalg import LinearOperator, gmres
    u = u_old.copy()
    C, N = u.shape
    r0 = None
    for _ in range(max_it):
        r = O.residual(mesh, P, T, u, [u_old], 2, advection=adv)
        nr = np.linalg.norm(r)
        r0 = nr if r0 is None else r0
        if nr <= tol_rel * r0 or nr < 1e-14:
            return u
        lin = u.copy()
        J = LinearOperator((C * N, C * N),
                           matvec=lambda v: O.jvp(mesh, P, T, lin, v.reshape(C, N), advection=adv).ravel())
        du, info = gmres(J, -r.ravel(), rtol=1e-13, atol=0.0, restart=300, maxiter=50)
        u = u + du.reshape(C, N)
    raise RuntimeError("CPU Newton did not converge")


@pytest.mark.parametrize("prec", [64, 32])
def test_newton_with_advection_matches_cpu_newton(prec):
    import hpsint_b200 as hb
    cells, G, dt = (40, 20), 2, 1e-2
    u_old = _two_particles(cells)
    seg, data = _two_particle_advection(cells)
    adv = (seg, data, (0.0, 0.0, 0.0))
    mesh = oracle_mesh(2, cells)
    P = O.make_params(G, tensorial=True)
    T = O.make_time(1.0 / dt, 1.0, [-1.0 / dt])
    ref = _cpu_newton(mesh, P, T, u_old, adv)
    op = hb.SinteringOperatorGeneric(hb.Mesh(2, tuple(cells) + (1,)), hb.Params(G, tensorial=True))
    op.set_time_weights(1.0 / dt, [-1.0 / dt], 1.0)
    set_adv(op, seg, data)
    old = op.to_device(u_old)
    u = old.clone()
    st = hb.DampedNewtonSolver(op, hb.NonLinearData(nl_rel_tol=1e-10, nl_abs_tol=1e-16, l_rel_tol=1e-4,
                                                    nl_max_iter=20, inner_precision=prec)).solve(u, [old])
    torch.cuda.synchronize()
    assert st.status == 0
    assert np.max(np.abs(op.to_host(u) - ref)) < (1e-7 if prec == 64 else 1e-6)
    # advection moved the step away from the plain one
    plain = O.residual(mesh, P, T, ref, [u_old], 2)
    assert np.linalg.norm(plain) > 1e-3 * np.linalg.norm(O.residual(mesh, P, T, u_old, [u_old], 2))


@pytest.mark.parametrize("prec", [64, 32])
def test_graph_replayed_solve_reads_the_current_velocities(prec):
    """The second solve replays the GMRES graphs captured in the first one;
    new velocities in the same tables must give bitwise the result of a
    fresh context.  Both compared solves start with a cleared Newton history,
    so both build the preconditioner (which carries the advection terms) from
    the new velocities at their first iteration."""
    import hpsint_b200 as hb
    cells, G, dt = (40, 20), 2, 1e-2
    u_old = _two_particles(cells)
    seg, data = _two_particle_advection(cells)
    data2 = data.copy()
    data2[0, 0], data2[1, 5] = -1.5, -0.4

    def solve(op, d, clear=False):
        set_adv(op, seg, d)
        old = op.to_device(u_old)
        u = old.clone()
        newton = hb.DampedNewtonSolver(op, hb.NonLinearData(nl_rel_tol=1e-9, nl_abs_tol=1e-16,
                                                            inner_precision=prec))
        if clear:
            newton.clear()
        st = newton.solve(u, [old])
        torch.cuda.synchronize()
        assert st.status == 0
        return u

    def new_op():
        op = hb.SinteringOperatorGeneric(hb.Mesh(2, tuple(cells) + (1,)), hb.Params(G, tensorial=True))
        op.set_time_weights(1.0 / dt, [-1.0 / dt], 1.0)
        return op

    op = new_op()
    solve(op, data)
    solve(op, data)  # graphs captured by now
    replayed = solve(op, data2, clear=True)
    fresh_op = new_op()
    solve(fresh_op, data2)
    fresh = solve(fresh_op, data2, clear=True)
    assert torch.equal(replayed, fresh)


# --- the advection mechanism: forces from the state, velocities from forces

MECH = dict(k=2.5, cgb=0.0, ceq=0.9, smoothening=0.0, mt=0.3, mr=0.2)


def set_mech(op, seg, centers, **kw):
    prm = dict(MECH, **kw)
    op.set_advection_mechanism(torch.from_numpy(seg).cuda().contiguous(),
                               torch.from_numpy(np.ascontiguousarray(centers)).cuda().contiguous(), **prm)
    return prm


MECH_CASES = [
    # dim, cells, G, cgb, smoothening
    (2, (37, 21), 4, 0.0, 0.0),
    (2, (30, 26), 9, 0.14, 40.0),
    (3, (13, 11, 9), 5, 0.14, 0.0),
    (3, (11, 9, 10), 9, 0.0, 0.0),
]


@pytest.mark.parametrize("case", MECH_CASES, ids=[f"{c[0]}d-G{c[2]}-cgb{c[3]}-s{c[4]}" for c in MECH_CASES])
def test_forces_and_velocities_match_oracle(case):
    dim, cells, G, cgb, sm = case
    op, p, om = make_op(dim, cells, G, True)
    u = particle_state(dim, cells, G, seed=61)
    seg, data = advection_data(dim, cells, G, seed=62, n_seg_per_grain=3)
    centers = data[:, 6:9].copy()
    prm = set_mech(op, seg, centers, cgb=cgb, smoothening=sm)
    ud = op.to_device(u)
    vft = op.advection_forces(ud).cpu().numpy()
    ref = O.advection_forces(om, p, u, seg, centers, ORIGIN, prm["k"], cgb, prm["ceq"], sm)
    scale = np.abs(ref).max(axis=0, keepdims=True)
    assert np.all(np.abs(vft - ref) <= 1e-12 * scale + 1e-300)
    # the residual then moves the grains with the oracle's velocities for those forces
    table = O.advection_velocities(dim, ref, centers, prm["mt"], prm["mr"])
    op.set_time_weights(20.0, [-20.0], 1.0)
    r = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(r, ud, 2, [ud])
    op.fill_quadrature_point_values(ud)
    src = random_state(dim, cells, G, seed=63, smooth=False) - 0.5
    j = op.initialize_dof_vector()
    op.vmult(j, op.to_device(src))
    torch.cuda.synchronize()
    T = O.make_time(20.0, 1.0, [-20.0])
    adv = (seg, table, ORIGIN)
    assert block_rel_err(op.to_host(r), O.residual(om, p, T, u, [u], 2, advection=adv)) <= 1e-11
    assert block_rel_err(op.to_host(j), O.jvp(om, p, T, u, src, advection=adv)) <= 1e-11


def test_forces_under_the_cut_off_and_determinism():
    dim, cells, G = 3, (14, 9, 10), 6
    op, p, om = make_op(dim, cells, G, True)
    u = particle_state(dim, cells, G, seed=64)
    seg, data = advection_data(dim, cells, G, seed=65)
    centers = data[:, 6:9].copy()
    ud = op.to_device(u)
    op.set_component_mask(ud, 1e-3)
    prm = set_mech(op, seg, centers)
    a = op.advection_forces(ud)
    b = op.advection_forces(ud)
    torch.cuda.synchronize()
    assert torch.equal(a, b)  # fixed summation order
    ref = O.advection_forces(om, p, u, seg, centers, ORIGIN, prm["k"], 0.0, prm["ceq"], 0.0,
                             mask=O.grain_mask(om, p, u, 1e-3))
    scale = np.abs(ref).max(axis=0, keepdims=True)
    assert np.all(np.abs(a.cpu().numpy() - ref) <= 1e-12 * scale + 1e-300)


def test_segments_spanning_many_tiles():
    """One segment per grain over the whole mesh: the per-segment sums run
    over hundreds of tiles of the sorted item list."""
    dim, cells, G = 3, (40, 36, 30), 3
    op, p, om = make_op(dim, cells, G, False)
    u = particle_state(dim, cells, G, seed=66)
    n_cells = int(np.prod(cells))
    seg = np.repeat(np.arange(G, dtype=np.int32)[:, None], n_cells, axis=1)
    seg[1, ::7] = -1  # holes
    centers = np.array([[10.0, 12.0, 9.0], [25.0, 20.0, 15.0], [30.0, 5.0, 20.0]])
    prm = set_mech(op, seg, centers)
    vft = op.advection_forces(op.to_device(u)).cpu().numpy()
    ref = O.advection_forces(om, p, u, seg, centers, ORIGIN, prm["k"], 0.0, prm["ceq"], 0.0)
    scale = np.abs(ref).max(axis=0, keepdims=True)
    assert np.all(np.abs(vft - ref) <= 1e-12 * scale + 1e-300)


def _mech_cpu_newton(mesh, P, T, u_old, seg, centers, prm, tol_rel=1e-12, max_it=40):
    """Newton on R(u; v(u)) with J v at frozen velocities, as the device solve."""
    from scipy.sparse.linalg import LinearOperator, gmres
    u = u_old.copy()
    C, N = u.shape
    r0 = None
    for _ in range(max_it):
        vft = O.advection_forces(mesh, P, u, seg, centers, (0, 0, 0), prm["k"], prm["cgb"], prm["ceq"],
                                 prm["smoothening"])
        adv = (seg, O.advection_velocities(2, vft, centers, prm["mt"], prm["mr"]), (0.0, 0.0, 0.0))
        r = O.residual(mesh, P, T, u, [u_old], 2, advection=adv)
        nr = np.linalg.norm(r)
        r0 = nr if r0 is None else r0
        if nr <= tol_rel * r0 or nr < 1e-14:
            return u
        lin = u.copy()
        J = LinearOperator((C * N, C * N),
                           matvec=lambda v: O.jvp(mesh, P, T, lin, v.reshape(C, N), advection=adv).ravel())
        du, info = gmres(J, -r.ravel(), rtol=1e-13, atol=0.0, restart=300, maxiter=50)
        u = u + du.reshape(C, N)
    raise RuntimeError("CPU Newton did not converge")


@pytest.mark.parametrize("prec", [64, 32])
def test_newton_with_the_mechanism_matches_cpu_newton(prec):
    import hpsint_b200 as hb
    cells, G, dt = (40, 20), 2, 1e-2
    u_old = _two_particles(cells)
    seg, data = _two_particle_advection(cells)
    centers = data[:, 6:9].copy()
    prm = dict(MECH, mt=5.0, mr=5.0)
    mesh = oracle_mesh(2, cells)
    P = O.make_params(G, tensorial=True)
    T = O.make_time(1.0 / dt, 1.0, [-1.0 / dt])
    ref = _mech_cpu_newton(mesh, P, T, u_old, seg, centers, prm)
    op = hb.SinteringOperatorGeneric(hb.Mesh(2, tuple(cells) + (1,)), hb.Params(G, tensorial=True))
    op.set_time_weights(1.0 / dt, [-1.0 / dt], 1.0)
    op.set_advection_mechanism(torch.from_numpy(seg).cuda(), torch.from_numpy(centers).cuda(), **prm)
    old = op.to_device(u_old)
    u = old.clone()
    st = hb.DampedNewtonSolver(op, hb.NonLinearData(nl_rel_tol=1e-10, nl_abs_tol=1e-16, l_rel_tol=1e-4,
                                                    nl_max_iter=30, inner_precision=prec)).solve(u, [old])
    torch.cuda.synchronize()
    assert st.status == 0
    assert np.max(np.abs(op.to_host(u) - ref)) < (1e-7 if prec == 64 else 1e-6)
    # the forces moved the grains: the step differs from the one without advection
    vft = op.advection_forces(u).cpu().numpy()
    assert np.abs(vft[:, 1:3]).max() > 0.0


def test_time_loop_with_tracked_segments():
    """TimeIntegrator with the advection mechanism: the particles of every
    order parameter become the segments before each step; the two grains
    approach faster than without advection and mass is conserved."""
    import hpsint_b200 as hb
    from hpsint_b200.time_integration import AdvectionData, TimeIntegrator
    cells, G = (48, 24), 2
    u0 = _two_particles(cells, R=7.0)
    dist = {}
    for adv in (None, AdvectionData(k=2.5, cgb=0.0, ceq=0.9, mt=5.0, mr=5.0)):
        op = hb.SinteringOperatorGeneric(hb.Mesh(2, tuple(cells) + (1,)), hb.Params(G, tensorial=True))
        ti = TimeIntegrator(op, advection=adv)
        ti.initialize(op.to_device(u0))
        u = ti.run(4, dt_schedule=[1e-2] * 4)
        torch.cuda.synchronize()
        uh = op.to_host(u)
        wx, wy = np.ones(cells[0] + 1), np.ones(cells[1] + 1)
        wx[[0, -1]] = wy[[0, -1]] = 0.5
        w = np.outer(wy, wx).ravel()
        x = np.tile(np.arange(cells[0] + 1, dtype=float), cells[1] + 1)
        # eta-weighted centroids (the tracker's centers move in whole cells only)
        cx = [(w * uh[2 + b]) @ x / (w @ uh[2 + b]) for b in range(G)]
        dist[adv is None] = cx[1] - cx[0]
        # conserved to the Newton tolerance (the default nl_rel_tol 1e-5 of each step's initial residual)
        assert abs(w @ uh[0] - w @ u0[0]) <= 1e-6 * abs(w @ u0[0])
        if adv is not None:
            assert len(ti.advection_forces) == 4
            owners, vft = ti.advection_forces[-1]
            assert [o[0] for o in owners] == [0, 1] and vft.shape == (2, 4)
            assert vft[0, 1] > 0 > vft[1, 1]  # the grains pull towards each other
    assert dist[False] < dist[True] - 1e-4


@pytest.mark.parametrize("dim,cells,G", [(2, (37, 21), 4), (3, (13, 11, 9), 5)])
def test_courant_check_matches_oracle(dim, cells, G):
    op, p, om = make_op(dim, cells, G, True)
    seg, data = advection_data(dim, cells, G, seed=71, scale=3.0)
    set_adv(op, seg, data)
    diam = np.sqrt(sum(H[d] ** 2 for d in range(dim)))
    dt_crit = diam / max_speed(dim, cells, H, ORIGIN, seg, data)
    for f in (1 - 1e-9, 1 + 1e-9, 0.5, 2.0):
        dt = dt_crit * f
        assert op.check_courant(dt) == O.advection_courant(om, p, (seg, data, ORIGIN), dt) == (f < 1)
    # under the cut-off only the relevant grains count
    u = particle_state(dim, cells, G, seed=72)
    op.set_component_mask(op.to_device(u), 1e-3)
    mask = O.grain_mask(om, p, u, 1e-3)
    dt_m = diam / max_speed(dim, cells, H, ORIGIN, seg, data, mask)
    for f in (1 - 1e-9, 1 + 1e-9):
        assert op.check_courant(dt_m * f) == O.advection_courant(om, p, (seg, data, ORIGIN), dt_m * f, mask=mask)


def test_time_loop_halves_dt_on_courant_violation():
    import hpsint_b200 as hb
    from hpsint_b200.time_integration import AdvectionData, TimeIntegrationData, TimeIntegrator
    cells, G = (40, 20), 2
    op = hb.SinteringOperatorGeneric(hb.Mesh(2, tuple(cells) + (1,)), hb.Params(G, tensorial=True))
    # mt = mr = 50: velocities near 1, so the Courant limit sqrt(2) / |v| is near 1.5
    adv = AdvectionData(k=2.5, cgb=0.0, ceq=0.9, mt=50.0, mr=50.0, check_courant=True)
    ti = TimeIntegrator(op, td=TimeIntegrationData(time_step_init=4.0, time_step_min=1e-4), advection=adv)
    ti.initialize(op.to_device(_two_particles(cells)))
    ti.step()
    courant = [f for f in ti.failures if f[2] == -1]
    assert courant and ti.records[-1].dt <= 2.0


def test_rbm_golden_residual_on_gpu(goldens):
    """hpsint's residual_generic_*_rbm goldens through the device path: device
    tracker segments, device forces and velocities, advection kernels."""
    import hpsint_b200 as hb
    from hpsint_b200 import grain_tracker as GT
    from test_oracle_golden import agrees_to_digits, debug_case, rbm_segments
    a = goldens["rbm"]
    for tens, key in [(False, "residual_scalar_rbm"), (True, "residual_tensorial_rbm")]:
        mesh_o, P, T, u, perm = debug_case(goldens, tens)
        m = goldens["model"]
        op = hb.SinteringOperatorGeneric(
            hb.Mesh(2, (2, 1, 1)),
            hb.Params(2, m["A"], m["B"], m["kappa_c"], m["kappa_p"], m["Mvol"], m["Mvap"], m["Msurf"], m["Mgb"],
                      m["L"], tens))
        w0 = 1.0 / m["bdf1_dt"]
        op.set_time_weights(w0, [-w0], 1.0)
        ud = op.to_device(u)
        seg, centers, owners = GT.advection_segments(op, ud, a["threshold_lower"])
        op.set_advection_mechanism(seg, centers, a["k"], a["cgb"], a["ceq"], a["smoothening"], a["mt"], a["mr"])
        dst = op.initialize_dof_vector()
        op.evaluate_nonlinear_residual(dst, ud, 2, [ud.clone()])
        ours = op.to_host(dst)
        seg_o, cen_o = rbm_segments(mesh_o, u, a["threshold_lower"])
        assert np.array_equal(seg.cpu().numpy(), seg_o)
        vft = O.advection_forces(mesh_o, P, u, seg_o, cen_o, (0, 0, 0), a["k"], a["cgb"], a["ceq"], a["smoothening"])
        table = O.advection_velocities(2, vft, cen_o, a["mt"], a["mr"])
        ref = O.residual(mesh_o, P, T, u, [u.copy()], 2, advection=(seg_o, table, (0, 0, 0)))
        assert np.max(np.abs(ours - ref)) < 1e-9  # the BDF1 term cancels (w0 = 1e5): absolute bound
        assert agrees_to_digits(ours[:, perm], np.array(goldens[key]), goldens["residual_digits"])


@pytest.mark.parametrize("case", [CASES[0], CASES[1], CASES[3], CASES[5]],
                         ids=[ids(c) for c in (CASES[0], CASES[1], CASES[3], CASES[5])])
def test_preconditioner_with_advection_matches_oracle(case):
    """precondition_advection_ch / _ac: the block-Jacobi diagonals with the
    advection terms, full operator and under the cut-off's preconditioner."""
    import hpsint_b200 as hb
    dim, cells, G, tens = case
    op, p, om = make_op(dim, cells, G, tens)
    u = particle_state(dim, cells, G, seed=93)
    seg, data = advection_data(dim, cells, G, seed=94, scale=5.0)
    set_adv(op, seg, data)
    adv = (seg, data, ORIGIN)
    ud = op.to_device(u)
    op.set_time_weights(40.0, [-40.0], 1.0)
    op.fill_quadrature_point_values(ud)
    pc = hb.BlockPreconditioner2(op)
    T = O.make_time(40.0, 1.0, [-40.0])
    N = op.N
    for cut in (False, True):
        mask = None
        if cut:
            op.set_component_mask(ud, 1e-3)
            op.set_preconditioner_cut_off(True)
            mask = O.grain_mask(om, p, u, 1e-3)
        pc.do_update()
        ch = O.ch_blocks(om, p, T, u, mask=mask, advection=adv)
        assert block_rel_err(pc.ch_blocks()[:, :N].cpu().numpy(), ch) <= 1e-12
        inv = O.inverse_diagonal(O.ac_diagonal(om, p, T, u, mask=mask, advection=adv))
        assert block_rel_err(pc.inverse_diagonal()[:, :N].cpu().numpy(), inv) <= 1e-12
    # the terms are there: differ from the preconditioner without advection
    assert block_rel_err(ch, O.ch_blocks(om, p, T, u, mask=mask)) > 1e-8
