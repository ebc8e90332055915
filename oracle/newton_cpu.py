"""CPU restatement of the damped Newton-GMRES time step (test infrastructure
and the CPU leg of the benchmark; never part of the product path).

It follows the same algorithm the device solver restates, on the oracle's
residual, Jacobian-vector product and block-Jacobi diagonals (C++, OpenMP
over the host cores) with numpy BLAS-1, all in FP64:

  * DampedNewtonSolver::solve (lac/solvers_nonlinear.h:247-357): tau = 0.1,
    omega halved until |R(u + omega du)| < (1 - tau omega) |R(u)|, at most
    100 damping steps; convergence test NewtonSolverSolverControl::check
    (:92-117, absolute or relative to the initial residual, max_iter);
  * the preconditioner rebuild rule of setup_preconditioner
    (time_integration/time_marching.h:168-207): rebuild when the solver's
    Newton-iteration count is a multiple of threshold_newton_iter or the last
    solve took more than threshold_linear_iter GMRES iterations;
  * deal.II SolverGMRES (left preconditioning, restart, classical
    Gram-Schmidt with the re-orthogonalisation test of solvers_linear.h /
    solvers_linear_parameters.h:24: a second pass from the first iteration
    whose norm drops below 10 sqrt(eps) of its value before the pass), with
    ReductionControl(l_max_iter, l_abs_tol, l_rel_tol);
  * BlockPreconditioner2 with point-block Jacobi: 2x2 node blocks of the
    Cahn-Hilliard tangent and the Allen-Cahn inverse diagonal
    (sintering/preconditioners.h:1222-1283).
"""
import numpy as np

from . import oracle as O


class BlockJacobi:
    """z = blockdiag(CH 2x2 blocks^-1, AC diagonal^-1) r at the linearisation point."""

    def __init__(self, mesh, params, time, lin, threads=0):
        ch = O.ch_blocks(mesh, params, time, lin, threads)
        a, b, c, d = ch
        det = a * d - b * c
        scale = np.abs(a * d) + np.abs(b * c)
        ok = (det != 0.0) & np.isfinite(det) & (np.abs(det) > 1e-14 * scale)
        inv_det = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
        # a singular block falls back to the guarded point inverse (operator_base.h:386-388)
        pa = np.where(np.abs(a) > 1e-10, 1.0 / np.where(np.abs(a) > 1e-10, a, 1.0), 1.0)
        pd = np.where(np.abs(d) > 1e-10, 1.0 / np.where(np.abs(d) > 1e-10, d, 1.0), 1.0)
        self.i00 = np.where(ok, d * inv_det, pa)
        self.i01 = np.where(ok, -b * inv_det, 0.0)
        self.i10 = np.where(ok, -c * inv_det, 0.0)
        self.i11 = np.where(ok, a * inv_det, pd)
        self.ac = O.inverse_diagonal(O.ac_diagonal(mesh, params, time, lin, threads))

    def apply(self, r):
        z = np.empty_like(r)
        z[0] = self.i00 * r[0] + self.i01 * r[1]
        z[1] = self.i10 * r[0] + self.i11 * r[1]
        z[2:] = self.ac * r[2:]
        return z


class ChSGS(BlockJacobi):
    """Block 0 (c, mu) by one multicolour symmetric Gauss-Seidel sweep pair on
    the assembled Cahn-Hilliard block (oracle_ch_sgs), block 1 (the grains) by
    the Allen-Cahn inverse diagonal."""

    def __init__(self, mesh, params, time, lin, threads=0):
        super().__init__(mesh, params, time, lin, threads)
        self.mesh = mesh
        self.A = O.ch_matrix(mesh, params, time, lin, threads)

    def apply(self, r):
        z = np.empty_like(r)
        z[:2] = O.ch_sgs(self.mesh, self.A, r[:2])
        z[2:] = self.ac * r[2:]
        return z


def gmres(matvec, prec, b, restart=30, max_iter=1000, abs_tol=1e-10, rel_tol=1e-2, right=False):
    """Left-preconditioned restarted GMRES, x0 = 0 (right=True: right
    preconditioning, J P^-1 y = b, x = P^-1 y, so the Arnoldi residual is the
    true one).  Returns (x, iterations); raises RuntimeError when max_iter is
    reached."""
    if right:
        y, its = gmres(lambda v: matvec(prec(v)), lambda v: v, b, restart, max_iter, abs_tol, rel_tol)
        return prec(y), its
    x = np.zeros_like(b)
    its, tol, first, reorth = 0, 0.0, True, False
    thresh2 = 100.0 * np.finfo(np.float64).eps
    shape = b.shape
    while True:
        w = prec(b if first else b - matvec(x))
        beta = float(np.linalg.norm(w))
        if first:
            tol = max(abs_tol, rel_tol * beta)
            first = False
        if beta <= tol:
            return x, its
        if its >= max_iter:
            raise RuntimeError("GMRES: maximum number of iterations reached")
        V = np.empty((restart + 1, w.size))
        V[0] = w.ravel() / beta
        H = np.zeros((restart + 1, restart))
        cs, sn = np.zeros(restart), np.zeros(restart)
        g = np.zeros(restart + 1)
        g[0] = beta
        k, res = 0, beta
        for j in range(restart):
            w = prec(matvec(V[j].reshape(shape))).ravel()
            norm_before2 = float(w @ w)
            Vm = V[:j + 1]
            h = Vm @ w
            w = w - Vm.T @ h
            norm2 = float(w @ w)
            if not reorth and norm2 < thresh2 * norm_before2:
                reorth = True
            if reorth:
                h2 = Vm @ w
                w = w - Vm.T @ h2
                h = h + h2
                norm2 = float(w @ w)
            hn = np.sqrt(norm2)
            H[:j + 1, j] = h
            H[j + 1, j] = hn
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            r = np.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = H[j, j] / r, H[j + 1, j] / r
            H[j, j] = r
            H[j + 1, j] = 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            res = abs(g[j + 1])
            its += 1
            k = j + 1
            if res <= tol or its >= max_iter:
                break
            V[j + 1] = w / hn
        y = np.linalg.solve(np.triu(H[:k, :k]), g[:k])
        x = x + (V[:k].T @ y).reshape(shape)
        if res <= tol:
            return x, its
        if its >= max_iter:
            raise RuntimeError("GMRES: maximum number of iterations reached")


class NewtonCPU:
    """Damped Newton-GMRES for the BDF step R(u) = 0 of the oracle's operator."""

    def __init__(self, mesh, params, threads=0, nl_max_iter=10, nl_abs_tol=1e-20, nl_rel_tol=1e-5,
                 l_max_iter=1000, l_abs_tol=1e-10, l_rel_tol=1e-2, restart=30, threshold_newton_iter=100,
                 threshold_linear_iter=20, preconditioner=BlockJacobi, right_preconditioning=False):
        self.mesh, self.params, self.threads = mesh, params, threads
        self.pc_class = preconditioner
        self.nl = dict(max_iter=nl_max_iter, abs_tol=nl_abs_tol, rel_tol=nl_rel_tol)
        self.l = dict(restart=restart, max_iter=l_max_iter, abs_tol=l_abs_tol, rel_tol=l_rel_tol,
                      right=right_preconditioning)
        self.thr_n, self.thr_l = threshold_newton_iter, threshold_linear_iter
        self.history_newton, self.last_linear, self.pc = 0, 0, None

    def clear(self):
        self.history_newton, self.last_linear = 0, 0

    def solve(self, time, u, hist):
        """Newton solve of R(u) = 0 (BDF weights in `time`, old solutions in
        `hist`), u updated in place.  Returns dict of iteration counts."""
        m, p, th = self.mesh, self.params, self.threads
        res = lambda v: O.residual(m, p, time, v, hist, 2, th)  # noqa: E731
        r = res(u)
        stats = dict(newton_iterations=0, linear_iterations=0, residual_evaluations=1)
        nr = n0 = float(np.linalg.norm(r))

        def check(step, v):
            if v > self.nl["abs_tol"] and v / n0 > self.nl["rel_tol"] and step < self.nl["max_iter"]:
                return 0
            return 1 if (v <= self.nl["abs_tol"] or v / n0 <= self.nl["rel_tol"]) else 2

        status, it = check(0, nr), 0
        while status == 0:
            lin = u.copy()
            if self.pc is None or self.history_newton % self.thr_n == 0 or self.last_linear > self.thr_l:
                self.pc = self.pc_class(m, p, time, lin, th)
            du, lits = gmres(lambda v: O.jvp(m, p, time, lin, v, th), self.pc.apply, -r, **self.l)
            stats["linear_iterations"] += lits
            self.last_linear = lits
            tau, omega, n_tmp = 0.1, 1.0, 0
            while True:
                trial = u + omega * du
                r = res(trial)
                stats["residual_evaluations"] += 1
                nn = float(np.linalg.norm(r))
                omega /= 2.0
                n_tmp += 1
                if not (nn >= (1.0 - tau * omega) * nr) or n_tmp >= 100:
                    break
            if not nn < (1.0 - tau * omega) * nr:
                raise RuntimeError("Maximum number of damping iterations of damp Netwon exceeded!")
            u[:] = trial
            nr = nn
            it += 1
            self.history_newton += 1
            status = check(it, nr)
        stats["newton_iterations"] = it
        if status != 1:
            raise RuntimeError("Maximum number of Newton iterations of damp Netwon exceeded!")
        return stats


def bdf1_steps(mesh, params, u0, dts, threads=0, **nl):
    """BDF1 steps with the given step sizes (mu weight 1); returns the final
    state and per-step statistics."""
    solver = NewtonCPU(mesh, params, threads, **nl)
    u = u0.copy()
    recs = []
    for dt in dts:
        T = O.make_time(1.0 / dt, 1.0, [-1.0 / dt])
        old = u.copy()
        recs.append(solver.solve(T, u, [old]))
    return u, recs
