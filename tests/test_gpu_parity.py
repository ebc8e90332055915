"""CUDA operator vs the CPU oracle (parity tests proper; need a B200).

Tolerances
  FP64 residual / Jacobian-vector product: per-block relative l2 error <= 1e-12
  FP32 Jacobian-vector product (FP32 accumulation): <= 2e-5 against the FP64
  oracle evaluated at the FP32-rounded inputs
  preconditioner diagonals: <= 1e-12
"""
import numpy as np
import pytest

from helpers import block_rel_err, n_nodes, oracle_mesh, random_state
from oracle import oracle as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def make_op(dim, cells, G, tensorial, h=(1.0, 1.0, 1.0), **kw):
    import hpsint_b200 as hb
    mesh = hb.Mesh(dim, tuple(cells) + (1,) * (3 - len(cells)), h)
    params = hb.Params(G, tensorial=tensorial, **kw)
    return hb.SinteringOperatorGeneric(mesh, params), params


def oracle_params(p):
    return O.make_params(p.n_grains, p.A, p.B, p.kappa_c, p.kappa_p, p.Mvol, p.Mvap, p.Msurf, p.Mgb, p.L,
                         p.tensorial)


CASES = [
    # dim, cells, G, tensorial, h
    (2, (11, 6), 2, True, (1.0, 1.0, 1.0)),
    (2, (11, 6), 2, False, (1.0, 1.0, 1.0)),
    (2, (17, 9), 5, True, (0.5, 0.7, 1.0)),
    (2, (8, 8), 1, True, (1.0, 1.0, 1.0)),
    (3, (5, 7, 3), 4, True, (1.0, 1.0, 1.0)),
    (3, (5, 7, 3), 4, False, (1.0, 1.0, 1.0)),
    (3, (8, 4, 4), 3, True, (0.8, 1.1, 0.9)),
    (3, (4, 4, 2), 1, False, (1.0, 1.0, 1.0)),
    (3, (6, 5, 5), 12, True, (1.0, 1.0, 1.0)),
    (2, (9, 10), 12, False, (1.0, 1.0, 1.0)),
]


def ids(c):
    return f"{c[0]}d-{'x'.join(map(str, c[1]))}-G{c[2]}-{'tens' if c[3] else 'scal'}"


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
@pytest.mark.parametrize("wtd", [0, 1, 2])
def test_residual_f64_matches_oracle(case, wtd):
    dim, cells, G, tens, h = case
    op, p = make_op(dim, cells, G, tens, h)
    u = random_state(dim, cells, G, seed=1)
    old = random_state(dim, cells, G, seed=2)
    old2 = random_state(dim, cells, G, seed=3)
    w = [11.0, -7.5, 3.5] if wtd == 2 else [10.0]
    hist = [old, old2] if wtd == 2 else []
    op.set_time_weights(w[0], w[1:] if wtd == 2 else [-w[0]], 1.0)
    dst = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(dst, op.to_device(u), wtd, [op.to_device(x) for x in hist])
    torch.cuda.synchronize()
    T = O.make_time(w[0], 1.0, w[1:] if wtd == 2 else [-w[0]])
    ref = O.residual(oracle_mesh(dim, cells, h), oracle_params(p), T, u, hist, wtd)
    assert block_rel_err(op.to_host(dst), ref) <= 1e-12


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_jvp_f64_matches_oracle(case):
    dim, cells, G, tens, h = case
    op, p = make_op(dim, cells, G, tens, h)
    lin = random_state(dim, cells, G, seed=4)
    src = random_state(dim, cells, G, seed=5, smooth=False) - 0.5
    op.set_time_weights(25.0, [-25.0], 1.0)
    op.fill_quadrature_point_values(op.to_device(lin))
    dst = op.initialize_dof_vector()
    op.vmult(dst, op.to_device(src))
    torch.cuda.synchronize()
    ref = O.jvp(oracle_mesh(dim, cells, h), oracle_params(p), O.make_time(25.0, 1.0, [-25.0]), lin, src)
    assert block_rel_err(op.to_host(dst), ref) <= 1e-12


@pytest.mark.skipif(not torch.cuda.is_available() or torch.cuda.device_count() < 2,
                    reason="needs two visible GPUs")
def test_jvp_on_two_devices_matches_oracle():
    """The launch set-up (shared-memory attributes, persistent grid size) is
    kept per device: a process that uses a second GPU first and then the
    first one gets correct products on both (3D, G = 4: more than 48 KB of
    dynamic shared memory per block)."""
    dim, cells, G, tens, h = 3, (5, 7, 3), 4, True, (1.0, 1.0, 1.0)
    lin = random_state(dim, cells, G, seed=4)
    src = random_state(dim, cells, G, seed=5, smooth=False) - 0.5
    for dev in (1, 0, 1):
        with torch.cuda.device(dev):
            op, p = make_op(dim, cells, G, tens, h)
            op.set_time_weights(25.0, [-25.0], 1.0)
            op.fill_quadrature_point_values(op.to_device(lin))
            dst = op.initialize_dof_vector()
            op.vmult(dst, op.to_device(src))
            torch.cuda.synchronize()
            ref = O.jvp(oracle_mesh(dim, cells, h), oracle_params(p), O.make_time(25.0, 1.0, [-25.0]), lin, src)
            assert dst.device.index == dev
            assert block_rel_err(op.to_host(dst), ref) <= 1e-12, dev


# The full FP32 product runs two tiles per block in packed pairs: odd tile
# counts (a lone last tile), partial tiles at the mesh's high faces in
# either lane, and the large-G one-block-per-SM instances.
F32_CASES = CASES[:6] + [
    (3, (9, 4, 2), 2, True, (1.0, 1.0, 1.0)),     # 3 tiles
    (3, (13, 5, 3), 5, False, (0.9, 1.0, 1.2)),   # 4 x 2 x 2 tiles, partial in x, y and z
    (3, (6, 5, 5), 12, True, (1.0, 1.0, 1.0)),
    (2, (25, 9), 3, True, (1.0, 1.0, 1.0)),       # 4 x 2 tiles, the last column partial
    (2, (9, 10), 12, False, (1.0, 1.0, 1.0)),
]


@pytest.mark.parametrize("case", F32_CASES, ids=[ids(c) for c in F32_CASES])
def test_jvp_f32_close_to_oracle(case):
    dim, cells, G, tens, h = case
    op, p = make_op(dim, cells, G, tens, h)
    lin = random_state(dim, cells, G, seed=6).astype(np.float32).astype(np.float64)
    src = (random_state(dim, cells, G, seed=7, smooth=False) - 0.5).astype(np.float32).astype(np.float64)
    op.set_time_weights(25.0, [-25.0], 1.0)
    op.fill_quadrature_point_values(op.to_device(lin))
    dst = op.initialize_dof_vector(torch.float32)
    op.vmult(dst, op.to_device(src, torch.float32))
    torch.cuda.synchronize()
    ref = O.jvp(oracle_mesh(dim, cells, h), oracle_params(p), O.make_time(25.0, 1.0, [-25.0]), lin, src)
    assert block_rel_err(op.to_host(dst), ref) <= 2e-5


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_preconditioner_matches_oracle(case):
    import hpsint_b200 as hb
    dim, cells, G, tens, h = case
    op, p = make_op(dim, cells, G, tens, h)
    lin = random_state(dim, cells, G, seed=8)
    op.set_time_weights(40.0, [-40.0], 1.0)
    op.fill_quadrature_point_values(op.to_device(lin))
    pc = hb.BlockPreconditioner2(op)
    pc.do_update()
    T = O.make_time(40.0, 1.0, [-40.0])
    om, opar = oracle_mesh(dim, cells, h), oracle_params(p)
    ch_ref = O.ch_blocks(om, opar, T, lin)
    ac_ref = O.ac_diagonal(om, opar, T, lin)
    N = op.N
    ch = pc.ch_blocks()[:, :N].cpu().numpy()
    inv = pc.inverse_diagonal()[:, :N].cpu().numpy()
    assert block_rel_err(ch, ch_ref) <= 1e-12
    assert block_rel_err(inv, O.inverse_diagonal(ac_ref)) <= 1e-12
    # apply: z = blockdiag(CH^-1, AC^-1) r
    r = random_state(dim, cells, G, seed=9, smooth=False) - 0.5
    z = op.initialize_dof_vector()
    pc.vmult(z, op.to_device(r))
    det = ch_ref[0] * ch_ref[3] - ch_ref[1] * ch_ref[2]
    zc = (ch_ref[3] * r[0] - ch_ref[1] * r[1]) / det
    zm = (-ch_ref[2] * r[0] + ch_ref[0] * r[1]) / det
    zref = np.vstack([zc, zm, O.inverse_diagonal(ac_ref) * r[2:]])
    assert block_rel_err(op.to_host(z), zref) <= 1e-12
    z32 = op.initialize_dof_vector(torch.float32)
    pc.vmult(z32, op.to_device(r, torch.float32))
    assert block_rel_err(op.to_host(z32), zref) <= 1e-5


def test_golden_debug_residual_on_gpu(goldens):
    """hpsint's residual_generic_*_no_rbm goldens through the CUDA kernels."""
    from test_oracle_golden import agrees_to_digits, debug_case
    import hpsint_b200 as hb
    for tens, key in [(False, "residual_scalar"), (True, "residual_tensorial")]:
        mesh_o, P, T, u, perm = debug_case(goldens, tens)
        m = goldens["model"]
        op = hb.SinteringOperatorGeneric(
            hb.Mesh(2, (2, 1, 1)),
            hb.Params(2, m["A"], m["B"], m["kappa_c"], m["kappa_p"], m["Mvol"], m["Mvap"], m["Msurf"], m["Mgb"],
                      m["L"], tens))
        w0 = 1.0 / m["bdf1_dt"]
        op.set_time_weights(w0, [-w0], 1.0)
        dst = op.initialize_dof_vector()
        ud = op.to_device(u)
        op.evaluate_nonlinear_residual(dst, ud, 2, [ud.clone()])
        ours = op.to_host(dst)
        ref = O.residual(mesh_o, P, T, u, [u.copy()], 2)
        # the BDF1 term cancels (w0 = 1e5): compare with an absolute bound
        assert np.max(np.abs(ours - ref)) < 1e-9
        assert agrees_to_digits(ours[:, perm], np.array(goldens[key]), goldens["residual_digits"])


def test_blas_reductions_match_numpy():
    import ctypes
    import hpsint_b200 as hb
    from hpsint_b200 import _lib as L
    op, _ = make_op(3, (5, 4, 3), 2, True)
    rng = np.random.default_rng(11)
    x = torch.tensor(rng.standard_normal((op.C, op.ld)), device="cuda")
    y = torch.tensor(rng.standard_normal((op.C, op.ld)), device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    n = op.C * op.ld
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    L.check(L.lib().sint_vec_dot_f64(op._h, n, x.data_ptr(), y.data_ptr(), out.data_ptr(), s), "dot")
    L.check(L.lib().sint_vec_norm2_f64(op._h, n, x.data_ptr(), out[1:].data_ptr(), s), "norm")
    xd, yd = x.cpu().numpy().ravel(), y.cpu().numpy().ravel()
    assert abs(out[0].item() - xd @ yd) <= 1e-12 * np.abs(xd * yd).sum()
    assert abs(out[1].item() - np.linalg.norm(xd)) <= 1e-13 * np.linalg.norm(xd)
    # determinism: same bits on a second call
    out2 = torch.zeros(1, dtype=torch.float64, device="cuda")
    L.check(L.lib().sint_vec_dot_f64(op._h, n, x.data_ptr(), y.data_ptr(), out2.data_ptr(), s), "dot")
    assert out2[0].item() == out[0].item()
    x32, y32 = x.float(), y.float()
    L.check(L.lib().sint_vec_dot_f32(op._h, n, x32.data_ptr(), y32.data_ptr(), out.data_ptr(), s), "dot32")
    ref32 = x32.double().cpu().numpy().ravel() @ y32.double().cpu().numpy().ravel()
    assert abs(out[0].item() - ref32) <= 1e-12 * np.abs(xd * yd).sum()
    # axpy / sadd / scale
    z = y.clone()
    L.check(L.lib().sint_vec_sadd_f64(n, 0.5, 2.0, x.data_ptr(), z.data_ptr(), s), "sadd")
    assert torch.allclose(z, 0.5 * y + 2.0 * x, rtol=0, atol=1e-14)


def test_kernel_results_are_deterministic():
    op, _ = make_op(3, (9, 6, 5), 4, True)
    lin = random_state(3, (9, 6, 5), 4, seed=12)
    src = random_state(3, (9, 6, 5), 4, seed=13)
    op.set_time_weights(10.0, [-10.0], 1.0)
    op.fill_quadrature_point_values(op.to_device(lin))
    s = op.to_device(src)
    a, b = op.initialize_dof_vector(), op.initialize_dof_vector()
    op.vmult(a, s)
    op.vmult(b, s)
    assert torch.equal(a, b)


def test_errors_are_reported():
    import hpsint_b200 as hb
    with pytest.raises(hb.SintError) as e:
        make_op(3, (4, 4, 4), 13, True)
    assert e.value.status_name == "SINT_ERR_GRAINS"
    op, _ = make_op(2, (4, 4), 2, True)
    with pytest.raises(hb.SintError) as e:
        op.vmult(op.initialize_dof_vector(), op.initialize_dof_vector())
    assert e.value.status_name == "SINT_ERR_NOT_READY"


def _residual_and_jvp_errors(dim, cells, G, tens, h, u, lin, src):
    op, p = make_op(dim, cells, G, tens, h)
    op.set_time_weights(10.0, [-10.0], 1.0)
    T = O.make_time(10.0, 1.0, [-10.0])
    M = oracle_mesh(dim, cells, h)
    dst = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(dst, op.to_device(u), 1, [])
    e_res = block_rel_err(op.to_host(dst), O.residual(M, oracle_params(p), T, u, [], 1))
    op.fill_quadrature_point_values(op.to_device(lin))
    op.vmult(dst, op.to_device(src))
    torch.cuda.synchronize()
    e_jvp = block_rel_err(op.to_host(dst), O.jvp(M, oracle_params(p), T, lin, src))
    return e_res, e_jvp


def test_grain_boundary_filter_near_its_threshold():
    """unit_vector_filter_2 (tensor.h:156-174) switches at |grad(eta_i - eta_j)|^2
    = 1e-20.  Grains 1 and 2 are faint (nodal values ~1e-9, exact to full
    relative precision), so the squared norms of their gradient difference
    spread over 5e-22 .. 5e-20 (64 % of the nodes above the threshold) and
    both branches are taken at many points."""
    dim, cells, G = 3, (8, 7, 6), 3
    mk = lambda seed: random_state(dim, cells, G, seed=seed)
    u, lin, src = mk(21), mk(22), mk(23) - 0.5
    for x in (u, lin):
        x[3] *= 1e-9
        x[4] *= 7e-10
    assert max(_residual_and_jvp_errors(dim, cells, G, True, (1.0, 1.0, 1.0), u, lin, src)) <= 1e-12


def test_steep_gradients_beyond_the_float_seed_range():
    """With cells of 1e-20 the squared gradient norms reach ~1e40: above
    2^126 the float reciprocal seed of the grain-boundary filter would flush
    to zero, above FLT_MAX the inverse square root seed overflows; the double
    path must take the exact division there and still match the oracle."""
    dim, cells, G = 3, (5, 4, 3), 3
    mk = lambda seed: random_state(dim, cells, G, seed=seed)
    u, lin, src = mk(24), mk(25), mk(26) - 0.5
    assert max(_residual_and_jvp_errors(dim, cells, G, True, (1e-20, 1e-20, 1e-20), u, lin, src)) <= 1e-12
