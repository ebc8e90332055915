"""The residual's range hooks in device form (needs a B200).

evaluate_nonlinear_residual(dst, src, pre_operation, post_operation) lets the
reference's Jacobian-free operator perturb the state and take a
finite-difference quotient inside the cell loop (lac/jacobian_operator.h:
160-232).  sint_residual_f64_hooks does the same as data:
dst = scale * (R(src + perturb_scale * perturb) - subtract).  Checked here:

  * the fused perturbation equals the residual of the materialised perturbed
    state to 1e-12 (the kernel forms src + a x with one rounding);
  * the fused epilogue is bitwise the plain residual followed by
    (R - subtract) * scale, on plain, periodic and cut-off meshes;
  * the whole finite-difference quotient in one call approximates the
    analytic Jacobian-vector product (scalar mobility: exact tangent);
  * src is left untouched; the advection mechanism with a perturbation is
    rejected.
"""
import numpy as np
import pytest

from helpers import block_rel_err, particle_state, random_state

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def make(dim, cells, G, tensorial=True):
    import hpsint_b200 as hb
    op = hb.SinteringOperatorGeneric(hb.Mesh(dim, tuple(cells) + (1,) * (3 - dim)), hb.Params(G, tensorial=tensorial))
    op.set_time_weights(50.0, [-50.0], 1.0)
    return op


CASES = [(2, (37, 21), 3), (3, (13, 11, 9), 4)]


@pytest.mark.parametrize("dim,cells,G", CASES)
@pytest.mark.parametrize("variant", ["plain", "periodic", "cut_off"])
def test_hooks_equal_the_unfused_steps(dim, cells, G, variant):
    op = make(dim, cells, G)
    u = op.to_device(particle_state(dim, cells, G, seed=31))
    old = op.to_device(particle_state(dim, cells, G, seed=32, width=1.2))
    x = op.to_device(random_state(dim, cells, G, seed=33, smooth=False) - 0.5)
    sub = op.to_device(random_state(dim, cells, G, seed=34, smooth=False))
    if variant == "periodic":
        op.set_periodicity([0])
    if variant == "cut_off":
        op.set_component_mask(u, 1e-3)
    a, scale = 1e-3, -7.5
    u_copy = u.clone()
    # fused perturbation against the materialised perturbed state
    fused, plain = op.initialize_dof_vector(), op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(fused, u, 2, [old], perturb=x, perturb_scale=a)
    op.evaluate_nonlinear_residual(plain, u + a * x, 2, [old])
    torch.cuda.synchronize()
    assert torch.equal(u, u_copy)  # src is not modified
    assert block_rel_err(op.to_host(fused), op.to_host(plain)) <= 1e-12
    # fused epilogue against the plain residual and the same two operations
    epi = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(epi, u, 2, [old], subtract=sub, scale=scale)
    op.evaluate_nonlinear_residual(plain, u, 2, [old])
    torch.cuda.synchronize()
    N = op.N
    assert torch.equal(epi[:, :N], ((plain - sub) * scale)[:, :N])
    # scale alone (subtract zero)
    op.evaluate_nonlinear_residual(epi, u, 2, [old], scale=scale)
    torch.cuda.synchronize()
    assert torch.equal(epi[:, :N], (plain * scale)[:, :N])


@pytest.mark.parametrize("dim,cells,G", CASES)
def test_finite_difference_quotient_in_one_call(dim, cells, G):
    op = make(dim, cells, G, tensorial=False)
    u = op.to_device(particle_state(dim, cells, G, seed=41))
    old = op.to_device(particle_state(dim, cells, G, seed=42, width=1.2))
    v = op.to_device(random_state(dim, cells, G, seed=43))
    r_u = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(r_u, u, 2, [old])
    delta = 1e-6
    fd = op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(fd, u, 2, [old], perturb=v, perturb_scale=delta, subtract=r_u, scale=1.0 / delta)
    op.fill_quadrature_point_values(u)
    jv = op.initialize_dof_vector()
    op.vmult(jv, v)
    torch.cuda.synchronize()
    assert block_rel_err(op.to_host(fd), op.to_host(jv)) <= 1e-4


def test_perturbation_with_the_advection_mechanism_is_rejected():
    import hpsint_b200 as hb
    dim, cells, G = 2, (20, 16), 2
    op = make(dim, cells, G)
    u = op.to_device(particle_state(dim, cells, G, seed=51))
    seg = torch.zeros((G, cells[0] * cells[1]), dtype=torch.int32, device="cuda")
    seg[1] = 1
    centers = torch.tensor([[5.0, 5.0, 0.0], [12.0, 8.0, 0.0]], dtype=torch.float64, device="cuda")
    op.set_advection_mechanism(seg, centers, 1.0, 0.0, 1.0, 0.0, 1.0, 1.0)
    dst = op.initialize_dof_vector()
    with pytest.raises(hb.SintError) as e:
        op.evaluate_nonlinear_residual(dst, u, 2, [u], perturb=u, perturb_scale=1e-3)
    assert e.value.status_name == "SINT_ERR_ARG"
    # the epilogue alone is fine with the mechanism
    op.evaluate_nonlinear_residual(dst, u, 2, [u], subtract=u, scale=2.0)
    torch.cuda.synchronize()
    assert np.isfinite(op.to_host(dst)).all()
