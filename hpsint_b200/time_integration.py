"""Implicit BDF time stepping around the device Newton solve.

Mirrors the parts of hpsint's time loop that decide what the hot path is
asked to do:
  TimeIntegratorData / BDF weights  time_integration/time_integrator_data.h:98-163,
                                    time_schemes.h:64-153
  SolutionHistory                   time_integration/solution_history.h:136-205
  predictor hook                    sintering/driver.h:2001-2058 (initial Newton iterate)
  failure -> dt halving, restore    sintering/driver.h:2163-2202, :2489-2505
  dt growth after "good" steps      sintering/driver.h:2239-2243, :2387-2409
  grain cut-off before each attempt sintering/driver.h:2212-2218
  advection: tracker segments, then  sintering/driver.h:1000-1030, :2205-2224 (the
    forces in every residual        tracker runs before the step), residual_wrapper.h:36-84
  defaults                          time_integration/time_integrator_parameters.h:32-36
The solution stays on the device; a step is one sint_newton_solve call (or
several after failures).
"""
import time
from dataclasses import dataclass, field, replace

import torch

from . import _lib as L
from .operator import DampedNewtonSolver, NonLinearData, SinteringOperatorGeneric, bdf_weights


@dataclass
class TimeIntegrationData:
    scheme_order: int = 1          # BDF order
    time_step_init: float = 1e-3
    time_step_min: float = 1e-5
    time_step_max: float = 1e2
    growth_factor: float = 1.2
    desirable_newton_iterations: int = 5
    desirable_linear_iterations: int = 100


@dataclass
class AdvectionData:
    """AdvectionData (sintering/parameters.h:719-745) plus the tracker's
    threshold_lower that defines the grain segments."""
    k: float = 20.0
    cgb: float = 0.1
    ceq: float = 1.0
    smoothening: float = 0.0
    mt: float = 1.0
    mr: float = 1.0
    threshold_lower: float = 0.01
    check_courant: bool = False   # CFLChecker before every step attempt (driver.h:2219-2226)


@dataclass
class StepRecord:
    t: float
    dt: float
    newton_iterations: int
    linear_iterations: int
    residual_evaluations: int
    failed_tries: int
    wall_s: float
    initial_residual: float = 0.0
    final_residual: float = 0.0
    accepted_wall_s: float = 0.0   # the successful attempt alone (wall_s includes failed tries)
    reference_residual: float = 0.0  # |R(u_n)| of the step when a predicted guess was measured against it
    preconditioner_setups: int = 0   # of the successful attempt
    predict_s: float = 0.0           # predictor call and its reference residual, successful attempt


class TimeIntegrator:
    """Advance u_t = ... with BDF and adaptive dt on the GPU.

    predictor(history, dts, dt) -> device tensor or None: optional initial
    Newton iterate for the step of size dt, given the last solutions
    (history[0] = u_n, history[1] = u_{n-1} once it exists) and the accepted
    steps (dts[0] = dt_{n-1} ...); the learned predictor plugs in here.  None
    means the previous solution (hpsint's "None" predictor).

    tolerance_base decides what Newton's relative tolerance is relative to:
      "initial_guess"  the residual at the initial iterate, as hpsint's
                       NewtonSolverSolverControl (solvers_nonlinear.h:92-117);
      "old_solution"   the residual at u_n under the new step's weights, i.e.
                       the initial residual of the unpredicted solve.  Every
                       predictor is then held to the same absolute stop
                       nl_rel_tol * |R(u_n)|, so a better guess can only save
                       iterations, never loosen the answer.  Without a
                       predictor the two rules coincide.

    grain_cut_off_tolerance != 0 (GrainCutOffTolerance, parameters.h:314)
    sets the operator's grain cut-off from u_n before every step attempt, as
    the driver does before make_step; a predicted guess keeps u_n on the DoFs
    the cut-off takes out of the system (they have no equation this step).

    advection (AdvectionData) enables the advection mechanism: before every
    step attempt the particles of every order parameter of u_n become the
    segments (device labelling), and every residual evaluation of the solve
    moves them with the forces of its own state.
    """

    def __init__(self, op: SinteringOperatorGeneric, nl: NonLinearData = None, td: TimeIntegrationData = None,
                 predictor=None, tolerance_base="initial_guess", grain_cut_off_tolerance=0.0,
                 advection: AdvectionData = None):
        if tolerance_base not in ("initial_guess", "old_solution"):
            raise ValueError(f"tolerance_base must be 'initial_guess' or 'old_solution', not {tolerance_base!r}")
        self.op = op
        self.nl = nl or NonLinearData()
        self.td = td or TimeIntegrationData()
        self.newton = DampedNewtonSolver(op, self.nl)
        self.predictor = predictor
        self.tolerance_base = tolerance_base
        self.grain_cut_off_tolerance = float(grain_cut_off_tolerance)
        self.cut_off_statistics = []  # per accepted step: cells per number of relevant grains
        self.advection = advection
        self.advection_forces = []    # per accepted step: (owners, volume/force/torque per segment at u_n+1)
        self._r = None
        self.history = []     # old solutions, most recent first (device tensors)
        self.dts = []         # accepted time steps, most recent first
        self.t = 0.0
        self.dt = self.td.time_step_init
        self.records = []
        self.failures = []    # (t, dt, status, message, newton its, linear its, |r0|, |r|) of failed attempts

    def initialize(self, u0):
        """Start a run from u0: forgets earlier steps and the Newton history
        that decides preconditioner rebuilds."""
        self.history = [u0.clone()]
        self.dts = []
        self.t = 0.0
        self.dt = self.td.time_step_init
        self.records = []
        self.newton.clear()

    def _halve_or_raise(self):
        self.dt *= 0.5
        self.newton.clear()
        if self.dt <= self.td.time_step_min:
            last = self.failures[-1]
            raise L.SintError(8, "TimeIntegrator.step",
                              f"Minimum timestep size exceeded, solution failed! (t = {self.t:.6g}, last "
                              f"Newton status {last[2]}: {last[3]})")

    def _set_advection(self):
        """Segments from u_n and the mechanism; False when the Courant check
        (AdvectionData.check_courant) fails at the current dt."""
        from .grain_tracker import advection_segments
        a = self.advection
        seg, centers, self._owners = advection_segments(self.op, self.history[0], a.threshold_lower)
        self.op.set_advection_mechanism(seg, centers, a.k, a.cgb, a.ceq, a.smoothening, a.mt, a.mr)
        if a.check_courant:
            self.op.advection_forces(self.history[0])
            return self.op.check_courant(self.dt)
        return True

    def _weights(self, dt):
        order = min(self.td.scheme_order, len(self.history))
        w = bdf_weights(order, [dt] + self.dts[:order - 1])
        return w[0], w[1:order + 1]

    def _stop_rule(self, wh):
        """NonLinearData for a predicted solve under tolerance_base."""
        if self.tolerance_base == "initial_guess":
            return None
        if self._r is None:
            self._r = self.op.initialize_dof_vector()
        hist = self.history[:len(wh)]
        self.op.evaluate_nonlinear_residual(self._r, self.history[0], 2, hist)
        ref = self.op.norm(self._r)
        self._reference_residual = ref
        return replace(self.nl, nl_abs_tol=max(self.nl.nl_abs_tol, self.nl.nl_rel_tol * ref), nl_rel_tol=0.0)

    def step(self, u_out=None):
        """One accepted time step; returns the new solution (device)."""
        tries = 0
        t0 = time.perf_counter()
        while True:
            t_try = time.perf_counter()
            w0, wh = self._weights(self.dt)
            self.op.set_time_weights(w0, wh, 1.0)
            if self.grain_cut_off_tolerance != 0.0:
                self.op.set_component_mask(self.history[0], self.grain_cut_off_tolerance)
            if self.advection is not None and not self._set_advection():
                # ExcCourantConditionViolated -> process_failure (driver.h:2219-2227, :2498-2501)
                tries += 1
                self.failures.append((self.t, self.dt, -1, "The Courant condition was violated. The advection "
                                      "velocity is too high.", 0, 0, 0.0, 0.0))
                self._halve_or_raise()
                continue
            t_pred = time.perf_counter()
            guess = self.predictor(self.history, self.dts, self.dt) if self.predictor else None
            if guess is not None and self.grain_cut_off_tolerance != 0.0:
                # DoFs outside the cut-off's reach have no equation this step: keep their old values
                self.op.cut_off_freeze(guess, self.history[0])
            self._reference_residual = 0.0
            data = self._stop_rule(wh) if guess is not None else None  # its norm waits for the guess
            t_pred = time.perf_counter() - t_pred if guess is not None else 0.0
            u = (guess if guess is not None else self.history[0]).clone()
            st = self.newton.solve(u, self.history[:len(wh)], raise_on_failure=False, data=data)
            if st.status == L.SINT_OK:
                break
            # process_failure: halve dt, restore the last good state, forget the
            # Newton history that decides preconditioner rebuilds
            tries += 1
            self.failures.append((self.t, self.dt, st.status, L.last_error(), st.newton_iterations,
                                  st.linear_iterations, st.initial_residual, st.final_residual))
            self._halve_or_raise()
        torch.cuda.synchronize()
        self.t += self.dt
        t1 = time.perf_counter()
        self.records.append(StepRecord(self.t, self.dt, st.newton_iterations, st.linear_iterations,
                                       st.residual_evaluations, tries, t1 - t0, st.initial_residual,
                                       st.final_residual, t1 - t_try, self._reference_residual,
                                       st.preconditioner_setups, t_pred))
        if self.grain_cut_off_tolerance != 0.0:
            self.cut_off_statistics.append(self.op.component_mask_statistics())
        if self.advection is not None:
            self.advection_forces.append((self._owners, self.op.advection_forces(u).cpu().numpy()))
        self.history.insert(0, u)
        self.dts.insert(0, self.dt)
        keep = max(2, self.td.scheme_order)  # predictors use the last two states
        self.history = self.history[:keep]
        self.dts = self.dts[:keep]
        good = (st.newton_iterations < self.td.desirable_newton_iterations and
                st.linear_iterations < self.td.desirable_linear_iterations)
        if good and self.td.growth_factor > 1.0:
            self.dt = min(self.dt * self.td.growth_factor, self.td.time_step_max)
        return u

    def run(self, n_steps, dt_schedule=None, keep_states=False):
        """n_steps accepted steps.  dt_schedule: replay these step sizes instead
        of the adaptive control (a failure then raises).  keep_states: return
        every accepted solution (device tensors) as well."""
        states = [self.history[0].clone()] if keep_states else None
        for i in range(n_steps):
            if dt_schedule is not None:
                self.dt = dt_schedule[i]
                min_dt = self.td.time_step_min
                self.td.time_step_min = dt_schedule[i]  # no halving below the schedule: fail instead
                try:
                    self.step()
                finally:
                    self.td.time_step_min = min_dt
            else:
                self.step()
            if keep_states:
                states.append(self.history[0].clone())
        return (self.history[0], states) if keep_states else self.history[0]
