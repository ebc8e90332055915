"""The Gauss-Seidel Cahn-Hilliard preconditioner on the GPU against the oracle
(needs a B200).

  * the assembled Cahn-Hilliard block equals the oracle's (oracle_ch_matrix)
    to 1e-12 per (neighbour, entry) row block, with and without the
    preconditioner's grain cut-off and advection terms;
  * the FP64 apply equals the oracle's multicolour sweeps on (c, mu) and the
    inverse diagonal on the grains to 1e-12; the FP32 apply to 1e-4;
  * the device Newton solve with it (right-preconditioned GMRES) converges to
    the CPU Newton's step, and needs fewer GMRES iterations than the
    block-Jacobi preconditioner with left preconditioning.
"""
import numpy as np
import pytest

from helpers import advection_data, block_rel_err, oracle_mesh, particle_state, random_state
from oracle import oracle as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

CASES = [
    # dim, cells, G, tensorial
    (2, (37, 21), 3, True),
    (2, (30, 26), 4, False),
    (3, (13, 11, 9), 4, True),
    (3, (9, 8, 7), 9, True),
    (3, (10, 9, 8), 2, False),
]


def ids(c):
    return f"{c[0]}d-G{c[2]}-{'tens' if c[3] else 'scal'}"


def make(dim, cells, G, tensorial):
    import hpsint_b200 as hb
    op = hb.SinteringOperatorGeneric(hb.Mesh(dim, tuple(cells) + (1,) * (3 - dim)), hb.Params(G, tensorial=tensorial))
    return op, O.make_params(G, tensorial=tensorial), oracle_mesh(dim, cells)


def setup(op, u, w0=1e3):
    import hpsint_b200 as hb
    op.set_time_weights(w0, [-w0], 1.0)
    op.fill_quadrature_point_values(op.to_device(u))
    pc = hb.BlockPreconditioner2(op, block_0="ch_gauss_seidel")
    pc.do_update()
    return pc


def matrix_err(ours, ref):
    nk = ref.shape[0]
    return block_rel_err(ours.reshape(nk * 4, -1), ref.reshape(nk * 4, -1))


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_matrix_and_apply_match_oracle(case):
    dim, cells, G, tens = case
    op, p, om = make(dim, cells, G, tens)
    u = particle_state(dim, cells, G, seed=21)
    pc = setup(op, u)
    T = O.make_time(1e3, 1.0, [-1e3])
    N = op.N
    A_ref = O.ch_matrix(om, p, T, u)
    assert matrix_err(pc.ch_matrix()[:, :, :N].cpu().numpy(), A_ref) <= 1e-12
    r = random_state(dim, cells, G, seed=22, smooth=False) - 0.5
    z = op.initialize_dof_vector()
    pc.vmult(z, op.to_device(r))
    zref = np.vstack([O.ch_sgs(om, A_ref, r[:2]), O.inverse_diagonal(O.ac_diagonal(om, p, T, u)) * r[2:]])
    assert block_rel_err(op.to_host(z), zref) <= 1e-12
    z32 = op.initialize_dof_vector(torch.float32)
    pc.vmult(z32, op.to_device(r, torch.float32))
    assert block_rel_err(op.to_host(z32), zref) <= 1e-4


@pytest.mark.parametrize("case", CASES[:3], ids=[ids(c) for c in CASES[:3]])
def test_matrix_with_cut_off_and_advection(case):
    dim, cells, G, tens = case
    op, p, om = make(dim, cells, G, tens)
    u = particle_state(dim, cells, G, seed=23)
    ud = op.to_device(u)
    seg, data = advection_data(dim, cells, G, seed=24, scale=0.5)
    op.set_advection(torch.from_numpy(seg).cuda().contiguous(), torch.from_numpy(data).cuda().contiguous())
    adv = (seg, data, (0.0, 0.0, 0.0))
    T = O.make_time(1e3, 1.0, [-1e3])
    pc = setup(op, u)
    N = op.N
    assert matrix_err(pc.ch_matrix()[:, :, :N].cpu().numpy(), O.ch_matrix(om, p, T, u, advection=adv)) <= 1e-12
    op.set_component_mask(ud, 1e-3)
    op.set_preconditioner_cut_off(True)
    pc.do_update()
    mask = O.grain_mask(om, p, u, 1e-3)
    ref = O.ch_matrix(om, p, T, u, mask=mask, advection=adv)
    assert matrix_err(pc.ch_matrix()[:, :, :N].cpu().numpy(), ref) <= 1e-12
    # the cut-off changed the matrix (a grain-boundary mobility term dropped)
    assert matrix_err(ref, O.ch_matrix(om, p, T, u, advection=adv)) > 1e-10


def test_periodic_mesh_is_rejected():
    import hpsint_b200 as hb
    op, p, om = make(2, (12, 10), 2, True)
    op.set_periodicity([0])
    op.set_time_weights(10.0, [-10.0], 1.0)
    op.fill_quadrature_point_values(op.to_device(particle_state(2, (12, 10), 2, seed=1)))
    op.set_preconditioner_type("ch_gauss_seidel")
    with pytest.raises(hb.SintError) as e:
        hb.BlockPreconditioner2(op).do_update()
    assert e.value.status_name == "SINT_ERR_ARG"


_REF = {}


def _cpu_step(u0, G, n, dt):
    """The CPU Newton's BDF1 step (block-Jacobi, converged to 1e-10), cached."""
    from oracle import newton_cpu as NC
    if "u" not in _REF:
        om, p = oracle_mesh(3, (n, n, n)), O.make_params(G, tensorial=True)
        ref = u0.copy()
        NC.NewtonCPU(om, p, nl_rel_tol=1e-10, nl_max_iter=30, l_rel_tol=1e-8).solve(
            O.make_time(1.0 / dt, 1.0, [-1.0 / dt]), ref, [u0])
        _REF["u"] = ref
    return _REF["u"]


def _packing(n=24):
    from hpsint_b200 import packings as P
    c, r, col = P.lognormal_packing_3d(n=n, n_spheres=4, median=n / 4.5, sigma=0.2, max_grains=6, seed=0)
    G = int(col.max()) + 1
    return P.initial_state(3, (n, n, n), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), c, r, col, width=2.0), G


@pytest.mark.parametrize("prec", [64, 32])
def test_newton_with_gauss_seidel_matches_cpu_newton(prec):
    import hpsint_b200 as hb
    n = 24
    u0, G = _packing(n)
    dt = 1e-3
    ref = _cpu_step(u0, G, n, dt)
    counts = {}
    for kind, right in (("block_jacobi", False), ("ch_gauss_seidel", True)):
        op = hb.SinteringOperatorGeneric(hb.Mesh(3, (n, n, n)), hb.Params(G, tensorial=True))
        op.set_preconditioner_type(kind)
        op.set_time_weights(1.0 / dt, [-1.0 / dt], 1.0)
        old = op.to_device(u0)
        u = old.clone()
        st = hb.DampedNewtonSolver(op, hb.NonLinearData(nl_rel_tol=1e-9, inner_precision=prec,
                                                        right_preconditioning=right)).solve(u, [old])
        torch.cuda.synchronize()
        assert st.status == 0 and st.final_residual <= 1e-9 * st.initial_residual
        assert np.max(np.abs(op.to_host(u) - ref)) < 1e-6
        counts[kind] = st.linear_iterations
    assert counts["ch_gauss_seidel"] < counts["block_jacobi"], counts
