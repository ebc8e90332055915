"""Host logic of the time integrator (no GPU): what it asks the operator to do
before each step attempt and how it reacts to failures, with the device
calls replaced by fakes.

Mirrors sintering/driver.h:2163-2243 and :2489-2505: the grain cut-off and,
with advection, the tracker's segments and the advection mechanism are set
from u_n before every attempt; a failed Courant check (driver.h:2219-2227)
or a failed Newton solve halves dt and retries from u_n; a dt at or below the
minimum raises.
"""
import numpy as np
import pytest
import torch

from hpsint_b200 import _lib as L
from hpsint_b200 import time_integration as TI


class FakeStats:
    def __init__(self, status):
        self.status = status
        self.newton_iterations = 2
        self.linear_iterations = 10
        self.residual_evaluations = 3
        self.preconditioner_setups = 1
        self.initial_residual = 1.0
        self.final_residual = 1e-9


class FakeNewton:
    """Fails while dt is above `fail_above`."""
    fail_above = np.inf

    def __init__(self, op, data):
        self.op = op

    def solve(self, u, history, raise_on_failure=True, data=None):
        ok = self.op.dt_of_weights <= FakeNewton.fail_above
        if ok:
            u += 1.0
        return FakeStats(L.SINT_OK if ok else 6)

    def clear(self):
        self.op.log.append("clear")


class FakeOp:
    """Records the calls; the Courant check passes below `courant_dt`."""

    def __init__(self, courant_dt=np.inf):
        self.log = []
        self.courant_dt = courant_dt
        self.dt_of_weights = None

    def set_time_weights(self, w0, wh, walg=1.0):
        self.dt_of_weights = 1.0 / w0
        self.log.append(("weights", round(1.0 / w0, 12)))

    def set_component_mask(self, u, tol):
        self.log.append(("mask", tol))

    def component_mask_statistics(self):
        return np.array([1, 2])

    def set_advection_mechanism(self, seg, centers, k, cgb, ceq, smoothening, mt, mr):
        self.log.append(("mechanism", int(seg.sum()), tuple(centers.shape), k, mt, mr))

    def advection_forces(self, u):
        self.log.append("forces")
        return torch.zeros((2, 4))

    def check_courant(self, dt):
        self.log.append(("courant", round(dt, 12)))
        return dt < self.courant_dt


@pytest.fixture
def fakes(monkeypatch):
    monkeypatch.setattr(TI, "DampedNewtonSolver", FakeNewton)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    import hpsint_b200.grain_tracker as GT
    monkeypatch.setattr(GT, "advection_segments",
                        lambda op, u, thr: (torch.ones((2, 6), dtype=torch.int32), torch.zeros((2, 3)), [(0, 0), (1, 0)]))
    FakeNewton.fail_above = np.inf
    yield


def test_courant_violation_halves_dt(fakes):
    op = FakeOp(courant_dt=0.3)
    adv = TI.AdvectionData(k=2.0, mt=3.0, mr=4.0, check_courant=True)
    ti = TI.TimeIntegrator(op, td=TI.TimeIntegrationData(time_step_init=1.0, time_step_min=1e-3, growth_factor=1.0),
                           advection=adv)
    ti.initialize(torch.zeros((4, 6), dtype=torch.float64))
    u = ti.step()
    # 1.0 and 0.5 violate the Courant condition, 0.25 passes
    assert [f[1] for f in ti.failures] == [1.0, 0.5] and all(f[2] == -1 for f in ti.failures)
    assert ti.records[-1].dt == 0.25 and ti.records[-1].failed_tries == 2
    assert [e for e in op.log if isinstance(e, tuple) and e[0] == "courant"] == [
        ("courant", 1.0), ("courant", 0.5), ("courant", 0.25)]
    # the mechanism was set from u_n before every attempt, with the data's parameters
    mech = [e for e in op.log if isinstance(e, tuple) and e[0] == "mechanism"]
    assert len(mech) == 3 and mech[0] == ("mechanism", 12, (2, 3), 2.0, 3.0, 4.0)
    assert float(u[0, 0]) == 1.0 and len(ti.advection_forces) == 1


def test_newton_failure_halves_dt_and_minimum_raises(fakes):
    op = FakeOp()
    ti = TI.TimeIntegrator(op, td=TI.TimeIntegrationData(time_step_init=0.8, time_step_min=1e-2, growth_factor=1.0),
                           grain_cut_off_tolerance=1e-5)
    ti.initialize(torch.zeros((4, 6), dtype=torch.float64))
    FakeNewton.fail_above = 0.25
    ti.step()
    assert [f[1] for f in ti.failures] == [0.8, 0.4] and ti.records[-1].dt == 0.2
    # the cut-off mask is set before every attempt
    assert [e for e in op.log if isinstance(e, tuple) and e[0] == "mask"] == [("mask", 1e-5)] * 3
    # initialize() and process_failure (twice) forget the Newton history
    assert op.log.count("clear") == 3
    FakeNewton.fail_above = 0.0
    with pytest.raises(L.SintError):
        ti.step()


def test_dt_grows_after_good_steps(fakes):
    op = FakeOp()
    ti = TI.TimeIntegrator(op, td=TI.TimeIntegrationData(time_step_init=0.1, growth_factor=1.5, time_step_max=0.2))
    ti.initialize(torch.zeros((4, 6), dtype=torch.float64))
    ti.run(3)
    assert [r.dt for r in ti.records] == [0.1, pytest.approx(0.15), 0.2]
