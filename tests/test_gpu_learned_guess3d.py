"""The 3D learned guess end to end on a small case (GPU): FP64 trajectories
of two 32^3 lognormal packings, a short Adam run of the 3x3x3 net on 16^3
windows, then a held-out packing solved without a guess, with hpsint's
Linear predictor and with the learned guess (whole-mesh inference in depth
slabs smaller than the mesh, so the slab halos are exercised).  Every arm
converges to the same absolute Newton tolerance, so the answers must agree
to 1e-6 in max norm whatever the guess."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained3d():
    from hpsint_b200 import learned_guess as LG
    from hpsint_b200 import learned_guess3d as LG3
    from hpsint_b200.predictor import NetConfig
    return LG3.train_learned_guess3d([5, 6], n=32, n_spheres=6, n_steps=12, median=6.0, max_grains=6,
                                     net_cfg=NetConfig(dim=3, width=8, layers=3, seed=0),
                                     train_cfg=LG.TrainConfig(window=16, batch=2, iterations=150, log_every=25,
                                                              lr=2e-3))


def test_3d_training_reduces_the_loss(trained3d):
    _, _, _, info = trained3d
    hist = info["loss_history"]
    assert all(np.isfinite(l) and np.isfinite(b) for _, l, b in hist)
    assert hist[-1][1] < hist[0][1], hist


def test_3d_slab_inference_matches_one_window(trained3d):
    """Inference in depth slabs with halos equals one whole-mesh window (the
    halo covers the receptive field, so the slab seams change nothing)."""
    from hpsint_b200 import learned_guess3d as LG3
    net, norm, _, _ = trained3d
    case = LG3.make_case3d(9, n=32, n_spheres=6, median=6.0, max_grains=6)
    from hpsint_b200 import learned_guess as LG
    tr = LG.generate_trajectory(case, 3)
    hist, dts = [tr.states[-1], tr.states[-2]], [tr.dts[-1]]
    whole = LG3.LearnedPredictor3D(case.op, net, norm, slab=case.nodes, tensor_cores=False)
    slabs = LG3.LearnedPredictor3D(case.op, net, norm, slab=7, tensor_cores=False)
    a = whole(hist, dts, dts[0]).clone()
    b = slabs(hist, dts, dts[0])
    assert torch.allclose(a, b, rtol=0, atol=1e-6 * float(a.abs().max()))


def test_3d_learned_guess_keeps_the_answer(trained3d):
    from hpsint_b200 import learned_guess as LG
    from hpsint_b200 import learned_guess3d as LG3
    from hpsint_b200.operator import NonLinearData
    from hpsint_b200.time_integration import TimeIntegrationData, TimeIntegrator
    net, norm, _, _ = trained3d
    case = LG3.make_case3d(9, n=32, n_spheres=6, median=6.0, max_grains=6)
    out, schedule = {}, None
    for label, pred in (("plain", None), ("linear", LG.LinearPredictor(case.op)),
                        ("learned", LG3.LearnedPredictor3D(case.op, net, norm, slab=12)),
                        ("learned_safeguarded", LG3.LearnedPredictor3D(case.op, net, norm, slab=12, safeguard=True))):
        ti = TimeIntegrator(case.op, NonLinearData(nl_rel_tol=1e-8), TimeIntegrationData(time_step_init=1e-3),
                            predictor=pred, tolerance_base="old_solution")
        ti.initialize(case.u0)
        ti.run(8, dt_schedule=schedule)
        if schedule is None:
            schedule = [r.dt for r in ti.records]
        out[label] = (case.op.to_host(ti.history[0]), ti.records)
    ref = out["plain"][0]
    for label, (u, recs) in out.items():
        assert np.abs(u[0] - ref[0]).max() <= 1e-6 and np.abs(u[2:] - ref[2:]).max() <= 1e-6, label
        assert sum(r.failed_tries for r in recs) == 0, label
    newton = {k: sum(r.newton_iterations for r in v[1]) for k, v in out.items()}
    assert newton["learned_safeguarded"] <= newton["plain"], newton
