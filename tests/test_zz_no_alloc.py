"""The allocation-free Jacobian-vector product against the context-based one.

sint_jvp_f64_noalloc is for callers that may not call cudaMalloc (another
framework owns the memory pool, stream callbacks, fixed memory budgets): it
keeps its scratch in a fixed device array.  These checks call it through the
C ABI twice in a row (the shared scratch keeps the previous call's contents)
and compare with sint_jvp_f64 on a context holding the same state, within
the FP64 parity tolerance of the other tests (per-block relative 1e-12).
"""
import ctypes

import numpy as np
import pytest

from helpers import block_rel_err, random_state

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _noalloc(op, mesh, params, w0, w_alg, lin, src):
    from hpsint_b200 import _lib as L
    dst = op.initialize_dof_vector()
    rc = L.lib().sint_jvp_f64_noalloc(ctypes.byref(mesh.to_c()), ctypes.byref(params.to_c()), w0, w_alg,
                                       ctypes.c_void_p(lin.data_ptr()), ctypes.c_void_p(src.data_ptr()),
                                       ctypes.c_void_p(dst.data_ptr()),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    L.check(rc, "sint_jvp_f64_noalloc")
    torch.cuda.synchronize()
    return op.to_host(dst)


@pytest.mark.parametrize("dim,cells,G,tensorial", [(3, (12, 10, 8), 4, True), (2, (37, 21), 3, False),
                                                   (3, (9, 7, 5), 12, True)])
def test_noalloc_jvp_matches_context_jvp_twice(dim, cells, G, tensorial):
    import hpsint_b200 as hb
    mesh = hb.Mesh(dim, tuple(cells) + (1,) * (3 - dim))
    params = hb.Params(G, tensorial=tensorial)
    op = hb.SinteringOperatorGeneric(mesh, params)
    w0, w_alg = 30.0, 1.0
    op.set_time_weights(w0, [-w0], w_alg)
    lin = op.to_device(random_state(dim, cells, G, seed=21))
    op.fill_quadrature_point_values(lin)
    for call, seed in enumerate([22, 23]):
        src = op.to_device(random_state(dim, cells, G, seed=seed, smooth=False) - 0.5)
        ref = op.initialize_dof_vector()
        op.vmult(ref, src)
        torch.cuda.synchronize()
        ours = _noalloc(op, mesh, params, w0, w_alg, lin, src)
        assert block_rel_err(ours, op.to_host(ref)) <= 1e-12, f"call {call}"


def test_noalloc_at_the_largest_accepted_mesh_allocates_nothing():
    """64 x 64 x 36 cells at G = 4 need 16,588,800 bytes of tile-face
    partials, just inside the fixed array: the product still equals
    sint_jvp_f64 (an off-by-one in the scratch size would show at its end),
    one more layer of tiles is rejected, and repeated calls leave the
    device's free memory unchanged."""
    import hpsint_b200 as hb
    from hpsint_b200 import _lib as L
    dim, cells, G = 3, (64, 64, 36), 4
    mesh, params = hb.Mesh(dim, cells), hb.Params(G, tensorial=True)
    op = hb.SinteringOperatorGeneric(mesh, params)
    w0, w_alg = 30.0, 1.0
    op.set_time_weights(w0, [-w0], w_alg)
    lin = op.to_device(random_state(dim, cells, G, seed=31))
    op.fill_quadrature_point_values(lin)
    src = op.to_device(random_state(dim, cells, G, seed=32, smooth=False) - 0.5)
    ref = op.initialize_dof_vector()
    op.vmult(ref, src)
    torch.cuda.synchronize()
    ours = _noalloc(op, mesh, params, w0, w_alg, lin, src)
    assert block_rel_err(ours, op.to_host(ref)) <= 1e-12
    # no allocation: after a warm-up call, the free device memory stays put
    dst = op.initialize_dof_vector()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call():
        return L.lib().sint_jvp_f64_noalloc(ctypes.byref(mesh.to_c()), ctypes.byref(params.to_c()), w0, w_alg,
                                             ctypes.c_void_p(lin.data_ptr()), ctypes.c_void_p(src.data_ptr()),
                                             ctypes.c_void_p(dst.data_ptr()), stream)
    L.check(call(), "sint_jvp_f64_noalloc")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        L.check(call(), "sint_jvp_f64_noalloc")
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    # one more z-layer of tiles does not fit
    big = hb.Mesh(dim, (64, 64, 38))
    p = ctypes.c_void_p(dst.data_ptr())
    rc = L.lib().sint_jvp_f64_noalloc(ctypes.byref(big.to_c()), ctypes.byref(params.to_c()), w0, w_alg, p, p, p,
                                       None)
    assert L.STATUS_NAMES[rc] == "SINT_ERR_ARG"


def test_noalloc_rejects_meshes_beyond_its_scratch():
    import hpsint_b200 as hb
    from hpsint_b200 import _lib as L
    mesh = hb.Mesh(3, (128, 128, 128))
    params = hb.Params(4)
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    rc = L.lib().sint_jvp_f64_noalloc(ctypes.byref(mesh.to_c()), ctypes.byref(params.to_c()), 1.0, 1.0, p, p, p,
                                       None)
    assert L.STATUS_NAMES[rc] == "SINT_ERR_ARG"
    assert b"scratch" in L.lib().sint_last_error()
