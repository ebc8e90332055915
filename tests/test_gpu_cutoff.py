"""The grain cut-off on the GPU against the CPU oracle (needs a B200).

The masks must equal the oracle's bit for bit; the cut-off residual, Jacobian
products and preconditioner meet the same tolerances as the full operator
(FP64 1e-12 per-block relative, FP32 2e-5 against the oracle at FP32-rounded
inputs); switching the cut-off off gives back the full operator bit for bit.
States are packings of localised particles, so tiles and warps hold cells
with different grain sets.
"""
import numpy as np
import pytest

from helpers import block_rel_err, oracle_mesh, particle_state, random_state
from oracle import oracle as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def make_op(dim, cells, G, tensorial):
    import hpsint_b200 as hb
    mesh = hb.Mesh(dim, tuple(cells) + (1,) * (3 - len(cells)))
    params = hb.Params(G, tensorial=tensorial)
    return hb.SinteringOperatorGeneric(mesh, params), O.make_params(G, tensorial=tensorial)


CASES = [
    # dim, cells, G, tensorial, tolerance
    (2, (37, 21), 4, True, 1e-3),
    (2, (37, 21), 4, False, 1e-3),
    (2, (30, 26), 9, True, 1e-5),
    (3, (13, 11, 9), 5, True, 1e-3),
    (3, (13, 11, 9), 5, False, 1e-3),
    (3, (14, 9, 10), 10, True, 1e-5),
    (3, (9, 8, 7), 12, True, 0.2),
]


def ids(c):
    return f"{c[0]}d-G{c[2]}-{'tens' if c[3] else 'scal'}-tol{c[4]:g}"


def _mask_of(op):
    return op.get_component_mask().cpu().numpy().view(np.uint16)


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_mask_and_statistics_match_oracle(case):
    dim, cells, G, tens, tol = case
    op, p = make_op(dim, cells, G, tens)
    u = particle_state(dim, cells, G, seed=11)
    op.set_component_mask(op.to_device(u), tol)
    ref = O.grain_mask(oracle_mesh(dim, cells), p, u, tol)
    got = _mask_of(op)
    assert np.array_equal(got, ref)
    counts = np.bincount([bin(int(x)).count("1") for x in ref], minlength=G + 1)
    assert np.array_equal(op.component_mask_statistics(), counts)
    # the packing exercises mixed cells: several different grain counts
    assert np.count_nonzero(counts) >= 3


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_cut_off_residual_and_jacobian_match_oracle(case):
    dim, cells, G, tens, tol = case
    op, p = make_op(dim, cells, G, tens)
    om = oracle_mesh(dim, cells)
    u = particle_state(dim, cells, G, seed=12)
    old = particle_state(dim, cells, G, seed=12, width=1.2)
    src = random_state(dim, cells, G, seed=13, smooth=False) - 0.5
    ud = op.to_device(u)
    op.set_component_mask(ud, tol)
    mask = O.grain_mask(om, p, u, tol)
    op.set_time_weights(20.0, [-20.0], 1.0)
    T = O.make_time(20.0, 1.0, [-20.0])
    r = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(r, ud, 2, [op.to_device(old)])
    op.fill_quadrature_point_values(ud)
    j = op.initialize_dof_vector()
    op.vmult(j, op.to_device(src))
    torch.cuda.synchronize()
    r_ref = O.residual(om, p, T, u, [old], 2, mask=mask)
    j_ref = O.jvp(om, p, T, u, src, mask=mask)
    assert block_rel_err(op.to_host(r), r_ref) <= 1e-12
    assert block_rel_err(op.to_host(j), j_ref) <= 1e-12
    # the cut-off changed the result (it is not the full operator in disguise)
    assert block_rel_err(j_ref, O.jvp(om, p, T, u, src)) > 1e-9


@pytest.mark.parametrize("case", CASES[:4], ids=[ids(c) for c in CASES[:4]])
def test_cut_off_jacobian_f32_close_to_oracle(case):
    dim, cells, G, tens, tol = case
    op, p = make_op(dim, cells, G, tens)
    om = oracle_mesh(dim, cells)
    u = particle_state(dim, cells, G, seed=14).astype(np.float32).astype(np.float64)
    src = (random_state(dim, cells, G, seed=15, smooth=False) - 0.5).astype(np.float32).astype(np.float64)
    ud = op.to_device(u)
    op.set_component_mask(ud, tol)
    op.set_time_weights(20.0, [-20.0], 1.0)
    op.fill_quadrature_point_values(ud)
    j = op.initialize_dof_vector(torch.float32)
    op.vmult(j, op.to_device(src, torch.float32))
    torch.cuda.synchronize()
    j_ref = O.jvp(om, p, O.make_time(20.0, 1.0, [-20.0]), u, src, mask=O.grain_mask(om, p, u, tol))
    assert block_rel_err(op.to_host(j), j_ref) <= 2e-5


@pytest.mark.parametrize("case", CASES, ids=[ids(c) for c in CASES])
def test_cut_off_preconditioner_matches_oracle(case):
    import hpsint_b200 as hb
    dim, cells, G, tens, tol = case
    op, p = make_op(dim, cells, G, tens)
    om = oracle_mesh(dim, cells)
    u = particle_state(dim, cells, G, seed=16)
    ud = op.to_device(u)
    op.set_component_mask(ud, tol)
    mask = O.grain_mask(om, p, u, tol)
    op.set_time_weights(40.0, [-40.0], 1.0)
    op.fill_quadrature_point_values(ud)
    pc = hb.BlockPreconditioner2(op)
    T = O.make_time(40.0, 1.0, [-40.0])
    N = op.N
    # default: the block-Jacobi diagonals of the full operator; switched on:
    # the reference's cut-off assembly (preconditioners.h:787-817)
    for cut_pc, m in ((False, None), (True, mask)):
        op.set_preconditioner_cut_off(cut_pc)
        pc.do_update()
        assert block_rel_err(pc.ch_blocks()[:, :N].cpu().numpy(), O.ch_blocks(om, p, T, u, mask=m)) <= 1e-12
        inv_ref = O.inverse_diagonal(O.ac_diagonal(om, p, T, u, mask=m))
        assert block_rel_err(pc.inverse_diagonal()[:, :N].cpu().numpy(), inv_ref) <= 1e-12


def test_tolerance_zero_restores_the_full_operator_bitwise():
    dim, cells, G = 3, (13, 11, 9), 5
    op, p = make_op(dim, cells, G, True)
    u = particle_state(dim, cells, G, seed=17)
    src = op.to_device(random_state(dim, cells, G, seed=18, smooth=False) - 0.5)
    ud = op.to_device(u)
    op.set_time_weights(20.0, [-20.0], 1.0)
    op.fill_quadrature_point_values(ud)
    full = op.initialize_dof_vector()
    op.vmult(full, src)
    op.set_component_mask(ud, 1e-3)
    cut = op.initialize_dof_vector()
    op.vmult(cut, src)
    op.set_component_mask(ud, 0.0)
    again = op.initialize_dof_vector()
    op.vmult(again, src)
    torch.cuda.synchronize()
    assert not torch.equal(full, cut)
    assert torch.equal(full, again)
    with pytest.raises(Exception):
        op.component_mask_statistics()  # no cut-off set
    with pytest.raises(Exception):
        op.set_component_mask(ud, -1.0)


def test_newton_solve_with_cut_off():
    """A few implicit steps of a 2D packing with GrainCutOffTolerance 1e-5:
    the solves converge, mass is conserved to the Newton tolerance, and the
    states stay close to the full solve's (the cut terms are of the size of
    the tolerance)."""
    import hpsint_b200 as hb
    from hpsint_b200.time_integration import TimeIntegrator
    dim, cells, G = 2, (48, 40), 4
    u0 = particle_state(dim, cells, G, seed=19, width=2.0)
    out = {}
    for tol in (0.0, 1e-5):
        op, _ = make_op(dim, cells, G, True)
        ti = TimeIntegrator(op, grain_cut_off_tolerance=tol)
        ti.initialize(op.to_device(u0))
        dts = [1e-3 * 1.2 ** k for k in range(6)]
        u = ti.run(6, dt_schedule=dts)
        out[tol] = (op.to_host(u), ti)
    full, cut = out[0.0][0], out[1e-5][0]
    ti = out[1e-5][1]
    assert len(ti.cut_off_statistics) == 6
    stats = ti.cut_off_statistics[-1]
    assert stats.sum() == cells[0] * cells[1] and stats[:G].sum() > 0
    # integral of c (trapezoidal node weights = the Q1 mass lumping of int c)
    wx, wy = np.ones(cells[0] + 1), np.ones(cells[1] + 1)
    wx[[0, -1]] = wy[[0, -1]] = 0.5
    w = np.outer(wy, wx).ravel()
    # conserved to the Newton tolerance (relative 1e-8 of the initial residual), with or without the cut-off
    m0 = w @ u0[0]
    for u in (full, cut):
        assert abs(w @ u[0] - m0) <= 1e-8 * abs(m0)
    assert np.max(np.abs(cut - full)) <= 1e-3


@pytest.mark.parametrize("prec", [64, 32])
def test_skipping_zero_chunks_changes_nothing(prec):
    """Under the cut-off, GMRES skips the chunks of its vectors that no
    relevant cell reaches; the solves must be bitwise the same without it."""
    import hpsint_b200 as hb
    from hpsint_b200.time_integration import TimeIntegrationData, TimeIntegrator
    dim, cells, G = 3, (24, 20, 16), 5
    u0 = particle_state(dim, cells, G, seed=23, width=1.0)
    out = []
    for skip in (True, False):
        op, _ = make_op(dim, cells, G, True)
        op.set_cut_off_skip_zero_chunks(skip)
        ti = TimeIntegrator(op, hb.NonLinearData(inner_precision=prec), TimeIntegrationData(time_step_init=1e-4),
                            grain_cut_off_tolerance=1e-3)
        ti.initialize(op.to_device(u0))
        u = ti.run(4, dt_schedule=[1e-4] * 4)
        out.append((op.to_host(u), [(r.newton_iterations, r.linear_iterations) for r in ti.records],
                    ti.cut_off_statistics[-1]))
    assert out[0][2][0] > 0  # cells without any relevant grain exist
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.parametrize("dim,cells", [(2, (37, 21)), (3, (13, 11, 9))])
def test_cut_off_freeze_keeps_old_values_outside_the_cut(dim, cells):
    """Grain b at a node none of whose cells has b relevant gets no equation;
    cut_off_freeze puts the old value back there and touches nothing else."""
    G, tol = 5, 1e-3
    op, p = make_op(dim, cells, G, True)
    u_old = particle_state(dim, cells, G, seed=41)
    guess = u_old + 0.01 * (random_state(dim, cells, G, seed=42, smooth=False) - 0.5)
    op.set_component_mask(op.to_device(u_old), tol)
    g = op.to_device(guess)
    op.cut_off_freeze(g, op.to_device(u_old))
    got = op.to_host(g)
    # node activity from the oracle's cell masks
    mask = O.grain_mask(oracle_mesh(dim, cells), p, u_old, tol).reshape([cells[d] for d in reversed(range(dim))])
    node = np.zeros([cells[d] + 1 for d in reversed(range(dim))], dtype=np.uint16)
    for corner in range(1 << dim):
        sl = tuple(slice((corner >> (dim - 1 - a)) & 1, ((corner >> (dim - 1 - a)) & 1) + mask.shape[a])
                   for a in range(dim))
        node[sl] |= mask
    node = node.ravel()
    for b in range(G):
        live = ((node >> b) & 1).astype(bool)
        assert np.array_equal(got[2 + b][~live], u_old[2 + b][~live])
        assert np.array_equal(got[2 + b][live], guess[2 + b][live])
        assert (~live).any() and live.any()
    assert np.array_equal(got[:2], guess[:2])
