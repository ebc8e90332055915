"""Device damped Newton-GMRES (sint_newton_solve) on the GPU.

Reference solution: a CPU Newton iteration on the oracle's residual and
Jacobian-vector product with SciPy's GMRES, converged far below the test
tolerance.  Both solves converge to the same BDF1 step, so the final fields
must agree to the solver tolerances (max-norm 1e-7 for nl_rel_tol = 1e-10).
The FP32-inner solve (FP32 GMRES, Jacobian and preconditioner inside FP64
Newton) must reach the same FP64 Newton tolerance and agree with the FP64
solve to 1e-6.
"""
import numpy as np
import pytest

from helpers import oracle_mesh
from oracle import oracle as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def two_particle_state(cells=(40, 20), R=6.0, gap=-1.0, noise=0.0):
    from hpsint_b200 import packings as P
    nx, ny = cells
    c = np.array([[nx / 2 - R - gap / 2, ny / 2], [nx / 2 + R + gap / 2, ny / 2]])
    return P.initial_state(2, cells, (1.0, 1.0), (0.0, 0.0), c, np.array([R, R]), np.array([0, 1]), width=2.0,
                           noise=noise, seed=3)


def cpu_newton(mesh, P, T, u_old, tol_rel=1e-12, max_it=30):
    from scipy.sparse.linalg import LinearOperator, gmres
    u = u_old.copy()
    C, N = u.shape
    r0 = None
    for _ in range(max_it):
        r = O.residual(mesh, P, T, u, [u_old], 2)
        nr = np.linalg.norm(r)
        r0 = nr if r0 is None else r0
        if nr <= tol_rel * r0 or nr < 1e-14:
            return u
        lin = u.copy()
        J = LinearOperator((C * N, C * N), matvec=lambda v: O.jvp(mesh, P, T, lin, v.reshape(C, N)).ravel())
        du, info = gmres(J, -r.ravel(), rtol=1e-13, atol=0.0, restart=300, maxiter=50)
        u = u + du.reshape(C, N)
    raise RuntimeError("CPU Newton did not converge")


def gpu_solve(cells, G, u_old, dt, tensorial=True, **nl):
    import hpsint_b200 as hb
    op = hb.SinteringOperatorGeneric(hb.Mesh(2, tuple(cells) + (1,)), hb.Params(G, tensorial=tensorial))
    op.set_time_weights(1.0 / dt, [-1.0 / dt], 1.0)
    old = op.to_device(u_old)
    u = old.clone()
    data = hb.NonLinearData(**nl)
    st = hb.DampedNewtonSolver(op, data).solve(u, [old])
    torch.cuda.synchronize()
    return op.to_host(u), st


@pytest.mark.parametrize("tensorial", [True, False])
def test_newton_fp64_matches_cpu_newton(tensorial):
    cells, G, dt = (40, 20), 2, 1e-2
    u_old = two_particle_state(cells)
    mesh = oracle_mesh(2, cells)
    P = O.make_params(G, tensorial=tensorial)
    T = O.make_time(1.0 / dt, 1.0, [-1.0 / dt])
    ref = cpu_newton(mesh, P, T, u_old)
    ours, st = gpu_solve(cells, G, u_old, dt, tensorial, nl_rel_tol=1e-10, nl_abs_tol=1e-16, l_rel_tol=1e-4,
                         nl_max_iter=20)
    assert st.status == 0 and st.newton_iterations >= 1
    assert st.final_residual <= 1e-10 * st.initial_residual
    assert np.max(np.abs(ours - ref)) < 1e-7
    # the step moved the state (the comparison is not trivial)
    assert np.max(np.abs(ref - u_old)) > 1e-4


def test_newton_fp32_inner_matches_fp64():
    cells, G, dt = (48, 24), 2, 5e-2
    u_old = two_particle_state(cells, R=7.0)
    u64, s64 = gpu_solve(cells, G, u_old, dt, nl_rel_tol=1e-8, nl_abs_tol=1e-16, inner_precision=64)
    u32, s32 = gpu_solve(cells, G, u_old, dt, nl_rel_tol=1e-8, nl_abs_tol=1e-16, inner_precision=32)
    assert s64.status == 0 and s32.status == 0
    assert s32.final_residual <= 1e-8 * s32.initial_residual
    assert np.max(np.abs(u64 - u32)) < 1e-6


@pytest.mark.parametrize("prec", [64, 32])
def test_short_gmres_restart_reaches_the_same_step(prec):
    """GMRES(3): many restart cycles per Newton step, the same converged step as GMRES(30)."""
    u_old = two_particle_state(noise=1e-3)
    u30, s30 = gpu_solve((40, 20), 2, u_old, 1e-2, nl_rel_tol=1e-10, nl_abs_tol=1e-16, inner_precision=prec)
    u3, s3 = gpu_solve((40, 20), 2, u_old, 1e-2, nl_rel_tol=1e-10, nl_abs_tol=1e-16, inner_precision=prec,
                       gmres_restart=3, l_max_iter=5000)
    assert s30.status == 0 and s3.status == 0, (s30, s3)
    assert s3.linear_iterations > 3 * s3.newton_iterations  # restarts happened
    assert np.abs(u3 - u30).max() < 1e-7


@pytest.mark.parametrize("prec", [64, 32])
def test_graph_replayed_gmres_equals_a_fresh_solve(prec):
    """After a first solve the Arnoldi iterations replay captured CUDA graphs,
    updated when the time weights change; the result must be bitwise that of
    a fresh context solving the same step eagerly."""
    import hpsint_b200 as hb
    u_old = two_particle_state(noise=1e-3)
    data = hb.NonLinearData(nl_rel_tol=1e-10, nl_abs_tol=1e-16, inner_precision=prec)

    def solve(op, dt):
        op.set_time_weights(1.0 / dt, [-1.0 / dt], 1.0)
        old = op.to_device(u_old)
        u = old.clone()
        newton = hb.DampedNewtonSolver(op, data)
        newton.clear()  # same preconditioner-rebuild history as a fresh context
        st = newton.solve(u, [old])
        torch.cuda.synchronize()
        return op.to_host(u), st

    op = hb.SinteringOperatorGeneric(hb.Mesh(2, (40, 20, 1)), hb.Params(2))
    solve(op, 1e-2)                  # eager (first solve of this context)
    ua, sa = solve(op, 3e-3)         # graphs captured at dt = 3e-3
    ub, sb = solve(op, 7e-3)         # graphs updated for dt = 7e-3
    fresh_b, fsb = solve(hb.SinteringOperatorGeneric(hb.Mesh(2, (40, 20, 1)), hb.Params(2)), 7e-3)
    uc, sc = solve(op, 3e-3)         # back to dt = 3e-3
    assert sb.status == 0 and fsb.status == 0
    assert (sb.newton_iterations, sb.linear_iterations) == (fsb.newton_iterations, fsb.linear_iterations)
    assert np.array_equal(ub, fresh_b)
    assert np.array_equal(uc, ua)


def test_newton_3d_tensorial_converges():
    import hpsint_b200 as hb
    from hpsint_b200 import packings as P
    n, G = 16, 2
    cen = np.array([[n / 2 - 4.5, n / 2, n / 2], [n / 2 + 4.5, n / 2, n / 2]])
    u_old = P.initial_state(3, (n, n, n), (1, 1, 1), (0, 0, 0), cen, np.array([5.0, 5.0]), np.array([0, 1]))
    op = hb.SinteringOperatorGeneric(hb.Mesh(3, (n, n, n)), hb.Params(G))
    dt = 1e-2
    op.set_time_weights(1.0 / dt, [-1.0 / dt], 1.0)
    old = op.to_device(u_old)
    u = old.clone()
    st = hb.DampedNewtonSolver(op, hb.NonLinearData(nl_rel_tol=1e-8, inner_precision=32)).solve(u, [old])
    assert st.status == 0 and st.final_residual <= 1e-8 * st.initial_residual
    # the solution satisfies the FP64 residual it was solved for
    r = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(r, u, 2, [old])
    assert torch.linalg.norm(r).item() <= 1.01e-8 * st.initial_residual


def test_newton_failure_is_reported_not_raised_on_gpu():
    """ExcNewtonDidNotConverge as a status: one Newton iteration cannot reach 1e-14."""
    import hpsint_b200 as hb
    cells, G = (24, 12), 2
    u_old = two_particle_state(cells, R=4.0)
    op = hb.SinteringOperatorGeneric(hb.Mesh(2, cells + (1,)), hb.Params(G))
    op.set_time_weights(10.0, [-10.0], 1.0)
    old = op.to_device(u_old)
    u = old.clone()
    st = hb.DampedNewtonSolver(op, hb.NonLinearData(nl_max_iter=1, nl_rel_tol=1e-14, nl_abs_tol=0.0)).solve(
        u, [old], raise_on_failure=False)
    assert hb._lib.STATUS_NAMES[st.status] == "SINT_ERR_NEWTON"
    assert st.newton_iterations == 1
    # the context stays usable: a normal solve afterwards succeeds
    u2 = old.clone()
    st2 = hb.DampedNewtonSolver(op, hb.NonLinearData()).solve(u2, [old])
    assert st2.status == 0


def test_non_finite_state_fails_cleanly():
    """A NaN planted on the host before upload ends in a Newton failure status."""
    import hpsint_b200 as hb
    cells, G = (16, 8), 2
    u_old = two_particle_state(cells, R=3.0)
    bad = u_old.copy()
    bad[0, 5] = np.nan
    op = hb.SinteringOperatorGeneric(hb.Mesh(2, cells + (1,)), hb.Params(G))
    op.set_time_weights(10.0, [-10.0], 1.0)
    old = op.to_device(u_old)
    u = op.to_device(bad)
    st = hb.DampedNewtonSolver(op, hb.NonLinearData()).solve(u, [old], raise_on_failure=False)
    assert hb._lib.STATUS_NAMES[st.status] in ("SINT_ERR_NEWTON", "SINT_ERR_NO_CONVERGENCE")


def test_time_integrator_halves_dt_on_failure_and_grows_after_good_steps():
    """driver.h:2163-2202 / :2387-2409 semantics; the failure is injected on the
    host: the predictor's first initial guess carries a NaN."""
    import hpsint_b200 as hb
    from hpsint_b200.time_integration import TimeIntegrationData, TimeIntegrator
    cells, G = (32, 16), 2
    u0 = two_particle_state(cells, R=5.0)
    op = hb.SinteringOperatorGeneric(hb.Mesh(2, cells + (1,)), hb.Params(G))
    calls = []

    def poisoned_once(history, dts, dt):
        calls.append(dt)
        if len(calls) == 1:
            g = history[0].clone()
            g[0, 3] = float("nan")
            return g
        return None

    dt0 = 1e-3
    ti = TimeIntegrator(op, hb.NonLinearData(nl_rel_tol=1e-8), TimeIntegrationData(time_step_init=dt0),
                        predictor=poisoned_once)
    ti.initialize(op.to_device(u0))
    ti.run(3)
    r = ti.records
    assert r[0].failed_tries == 1 and r[0].dt == pytest.approx(dt0 / 2)
    assert calls[:2] == [dt0, dt0 / 2]
    for a, b in zip(r[:-1], r[1:]):
        good = a.newton_iterations < 5 and a.linear_iterations < 100
        assert b.dt == pytest.approx(a.dt * (1.2 if good else 1.0))
    # conservation of int c (natural boundary conditions): the c rows of the
    # residual sum to int (c - c_old) / dt, so int c_h = sum_n m_n c_n with the
    # row sums m_n of the mass matrix (half weight per boundary direction)
    wx = np.ones(cells[0] + 1)
    wx[[0, -1]] = 0.5
    wy = np.ones(cells[1] + 1)
    wy[[0, -1]] = 0.5
    m = np.outer(wy, wx).ravel()
    c0 = float(m @ u0[0])
    c1 = float(m @ ti.history[0][0, :op.N].cpu().numpy())
    assert abs(c1 - c0) <= 1e-6 * abs(c0)
