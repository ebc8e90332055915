"""The trained learned guess against the method without it and against
hpsint's own predictors (GPU).

A small version of the 2D many-grain workload: 128^2 cells, 12 circles,
three FP64 training trajectories, a short Adam run, then a held-out packing
solved by the plain FP64 method (previous-solution guess, hpsint's dt
control) and, on the same time grid, with hpsint's Linear, Euler and
Midpoint predictors and the learned guess.
All arms stop at the same absolute Newton tolerance (1e-8 relative to the
residual of the old solution), so the learned guess may only save iterations:
the final fields must agree with the plain run to 1e-6 in max norm."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    from hpsint_b200 import learned_guess as LG
    from hpsint_b200.predictor import NetConfig
    net, norm, tr, info = LG.train_learned_guess([11, 12, 13], n=128, n_circles=12, n_steps=40,
                                                 net_cfg=NetConfig(width=16, layers=4, seed=0),
                                                 train_cfg=LG.TrainConfig(window=48, batch=8, iterations=600,
                                                                          log_every=50))
    return net, norm, tr, info


def test_training_reduces_the_loss(trained):
    _, _, _, info = trained
    hist = info["loss_history"]
    assert info["triples"] >= 3 * 38
    assert all(np.isfinite(l) and np.isfinite(b) for _, l, b in hist)
    assert hist[-1][1] < 0.5 * hist[0][1], hist


def test_learned_guess_against_hpsint_predictors(trained):
    """The learned guess against hpsint's own predictors (Linear, Euler,
    Midpoint; driver.h:2005-2037) on a held-out packing, every arm on the
    plain run's time grid and converged to the same absolute tolerance:
    answers agree, the learned guess is closer to the converged step than the
    linear one (residual of the guess) and needs fewer GMRES iterations, with
    Newton iterations within one of the linear guess's."""
    from hpsint_b200 import learned_guess as LG
    net, norm, _, _ = trained
    case = LG.make_case(21, n=128, n_circles=12)
    res = LG.compare_arms(case, 30, net, norm,
                          arms=["fp64_plain", "fp64_linear", "fp64_euler", "fp64_midpoint", "fp64_learned",
                                "fp64_learned_safeguarded", "fp32_inner_learned_safeguarded"])
    for a, r in res.items():
        assert "failed" not in r, (a, r)
        assert r["max_abs_diff_c"] <= 1e-6 and r["max_abs_diff_eta"] <= 1e-6, (a, r)
        assert r["int_c_rel_change"] <= 1e-10, (a, r)
    plain, lin = res["fp64_plain"], res["fp64_linear"]
    # every predictor saves Newton iterations against the previous-solution guess
    for a in ("fp64_linear", "fp64_euler", "fp64_midpoint", "fp64_learned", "fp32_inner_learned_safeguarded"):
        assert res[a]["newton_iterations"] < plain["newton_iterations"], (a, res)
    for a in ("fp64_learned", "fp64_learned_safeguarded"):
        learned = res[a]
        assert learned["guess_residual_ratio_gmean"] < lin["guess_residual_ratio_gmean"], (a, res)
        assert learned["linear_iterations"] < lin["linear_iterations"], (a, res)
        assert learned["newton_iterations"] <= lin["newton_iterations"] + 1, (a, res)


def test_learned_predictor_matches_the_reference_network(trained):
    """Whole-mesh inference equals the NumPy network on the same features:
    FP32 kernels to 1e-4, the tensor-core (TF32) path to 2e-2 of the correction."""
    from hpsint_b200 import learned_guess as LG
    from oracle import predictor_ref as R
    net, norm, _, _ = trained
    case = LG.make_case(21, n=128, n_circles=12)
    tr = LG.generate_trajectory(case, 3)
    p = LG.LearnedPredictor(case.op, net, norm, tensor_cores=False)
    dt = tr.dts[2]
    guess = p([tr.states[2], tr.states[1]], [tr.dts[1]], dt).clone()
    p_tc = LG.LearnedPredictor(case.op, net, norm)  # inference on the tensor cores (TF32 products)
    guess_tc = p_tc([tr.states[2], tr.states[1]], [tr.dts[1]], dt).clone()
    net.check_tensor_cores()
    r = float(np.float32(dt / tr.dts[1]))  # the kernels take the step ratio as float
    G, nn = case.G, case.nodes
    un = case.op.to_host(tr.states[2]).reshape(2 + G, nn, nn)
    um = case.op.to_host(tr.states[1]).reshape(2 + G, nn, nn)
    sc, osc = p.scale.double().cpu().numpy(), p.oscale.double().cpu().numpy()
    # per-state scales: largest extrapolated increment of c, mu and the eta_i
    m = [np.abs(r * (un[0] - um[0])).max(), np.abs(r * (un[1] - um[1])).max(), np.abs(r * (un[2:] - um[2:])).max()]
    base = norm.base
    want_sc = [base[0], 1 / m[0], base[1], 1 / m[1], base[2], 1 / m[2]]
    want_osc = [base[3] / (m[0] * dt), base[4] / (m[1] * dt), base[5] / (m[2] * dt)]
    assert np.allclose(sc, want_sc, rtol=1e-6) and np.allclose(osc, want_osc, rtol=1e-6)
    xs = np.stack([un[0] * sc[0], r * (un[0] - um[0]) * sc[1], un[1] * sc[2], r * (un[1] - um[1]) * sc[3]])[None]
    xg = np.stack([np.stack([un[2 + g] * sc[4], r * (un[2 + g] - um[2 + g]) * sc[5]]) for g in range(G)])
    params = [{k: v.detach().double().cpu().numpy() for k, v in layer.items()} for layer in net.w]
    yg, ys, _ = R.forward(params, xg, xs, 1, G, net.cfg.slope)
    want = un + r * (un - um)
    want[0] += ys[0, 0] / osc[0]
    want[1] += ys[0, 1] / osc[1]
    want[2:] += yg[:, 0] / osc[2]
    got = case.op.to_host(guess).reshape(2 + G, nn, nn)
    # FP32 network: compare the predicted corrections relative to their size
    corr_ref, corr = want - (un + r * (un - um)), got - (un + r * (un - um))
    assert np.linalg.norm(corr - corr_ref) <= 1e-4 * np.linalg.norm(corr_ref) + 1e-12
    corr_tc = case.op.to_host(guess_tc).reshape(2 + G, nn, nn) - (un + r * (un - um))
    assert np.linalg.norm(corr_tc - corr_ref) <= 2e-2 * np.linalg.norm(corr_ref) + 1e-12
