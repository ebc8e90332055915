"""HostJvpPipeline: J v of pinned host vectors with copy-in, product and
copy-out of consecutive calls overlapped on three streams must give exactly
the products of the plain device call, in order, for every submitted call."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_pipelined_host_products_equal_device_products(depth):
    import hpsint_b200 as hb
    cells = (24, 20, 18)
    rng = np.random.default_rng(depth)
    G = 3
    op = hb.SinteringOperatorGeneric(hb.Mesh(3, cells), hb.Params(G))
    op.set_time_weights(50.0, [-50.0], 1.0)
    u = rng.uniform(0, 1, (G + 2, op.N))
    op.fill_quadrature_point_values(op.to_device(u))
    n_calls = 7
    srcs = [torch.zeros((op.C, op.ld), dtype=torch.float64).pin_memory() for _ in range(n_calls)]
    dsts = [torch.empty((op.C, op.ld), dtype=torch.float64).pin_memory() for _ in range(n_calls)]
    for s in srcs:
        s[:, :op.N] = torch.from_numpy(rng.uniform(-1, 1, (op.C, op.N)))
    pipe = hb.HostJvpPipeline(op, depth=depth)
    for d, s in zip(dsts, srcs):
        pipe.submit(d, s)
    pipe.synchronize()
    for d, s in zip(dsts, srcs):
        want = op.initialize_dof_vector()
        op.vmult(want, s.cuda())
        torch.cuda.synchronize()
        assert torch.equal(d, want.cpu())
