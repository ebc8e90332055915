"""Size-independent properties of the CUDA operator on the full operator-bench
state (128^3 cells, 8 spheres, G = 4, tensorial mobility, 12.9 M DoFs), where
the oracle would take minutes per product (needs a B200):

  * J(u) v is linear in v, in FP64 (1e-12) and FP32 (1e-4: the rounding of
    three FP32 products, each within 2e-5 of the exact one);
  * relabelling the grains of the state and of v permutes the eta rows of the
    residual and of J v and leaves the c and mu rows unchanged (1e-12; the
    free energy and the mobility are symmetric in the order parameters);
  * repeated products are bitwise identical (the tile-face sums are taken
    in a fixed order).

The file sorts last so that, under -x, nothing here can stop the parity
tests against the oracle from running.
"""
import numpy as np
import pytest

from helpers import block_rel_err

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

N_CELLS = 128


@pytest.fixture(scope="module")
def full():
    import hpsint_b200 as hb
    from hpsint_b200 import packings as P
    centers, radii, colours = P.operator_bench_packing(n=N_CELLS)
    G = int(colours.max()) + 1
    u = P.initial_state(3, (N_CELLS,) * 3, (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), centers, radii, colours, width=2.0,
                        noise=1e-3, seed=1)
    op = hb.SinteringOperatorGeneric(hb.Mesh(3, (N_CELLS,) * 3), hb.Params(G, tensorial=True))
    rng = np.random.default_rng(2)
    v1 = rng.uniform(-1.0, 1.0, u.shape)
    v2 = rng.uniform(-1.0, 1.0, u.shape)
    u_old = u + 0.02 * rng.uniform(-1.0, 1.0, u.shape)
    op.set_time_weights(1e3, [-1e3], 1.0)
    return dict(op=op, G=G, u=u, u_old=u_old, v1=v1, v2=v2)


def _jvp(op, ud, v):
    op.fill_quadrature_point_values(ud)
    dst = op.initialize_dof_vector(v.dtype)
    op.vmult(dst, v)
    return dst


def _relabel(x, perm):
    """New grain k = old grain perm[k] (rows 2.. of a (C, ld) block vector)."""
    y = x.clone()
    y[2:] = x[2:][torch.as_tensor(perm, device=x.device)]
    return y


def test_jvp_is_linear_in_v_at_full_size(full):
    op = full["op"]
    ud = op.to_device(full["u"])
    a, b = 0.75, -1.5
    for dtype, tol in ((torch.float64, 1e-12), (torch.float32, 1e-4)):
        v1, v2 = op.to_device(full["v1"], dtype), op.to_device(full["v2"], dtype)
        lhs = _jvp(op, ud, a * v1 + b * v2)
        rhs = a * _jvp(op, ud, v1) + b * _jvp(op, ud, v2)
        torch.cuda.synchronize()
        assert block_rel_err(op.to_host(lhs), op.to_host(rhs)) <= tol, dtype


def test_grain_relabelling_at_full_size(full):
    op, G = full["op"], full["G"]
    perm = np.roll(np.arange(G), 1)[::-1].copy()
    assert not np.array_equal(perm, np.arange(G))
    ud, uod, vd = op.to_device(full["u"]), op.to_device(full["u_old"]), op.to_device(full["v1"])
    up, uop, vp = _relabel(ud, perm), _relabel(uod, perm), _relabel(vd, perm)

    r, rp = op.initialize_dof_vector(), op.initialize_dof_vector()
    op.evaluate_nonlinear_residual(r, ud, 2, [uod])
    op.evaluate_nonlinear_residual(rp, up, 2, [uop])
    j = _jvp(op, ud, vd)
    jp = _jvp(op, up, vp)
    torch.cuda.synchronize()
    assert block_rel_err(op.to_host(rp), op.to_host(_relabel(r, perm))) <= 1e-12
    assert block_rel_err(op.to_host(jp), op.to_host(_relabel(j, perm))) <= 1e-12
    # and the relabelling is not a no-op on this state
    assert block_rel_err(op.to_host(_relabel(j, perm)), op.to_host(j)) > 1e-3


def test_repeated_products_are_bitwise_identical(full):
    op = full["op"]
    ud = op.to_device(full["u"])
    for dtype in (torch.float64, torch.float32):
        v = op.to_device(full["v1"], dtype)
        a = _jvp(op, ud, v)
        b = _jvp(op, ud, v)
        torch.cuda.synchronize()
        assert torch.equal(a, b), dtype
