"""C ABI checks that need no GPU: every declared symbol is exported, argument
validation, host-side defaults and the BDF weights."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "hpsint_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sint_\w+)\s*\(", txt)))


def test_header_declares_the_operator_interface():
    names = declared_functions()
    for required in ["sint_create", "sint_destroy", "sint_dof_layout", "sint_set_time_weights",
                     "sint_set_linearization_point", "sint_residual_f64", "sint_jvp_f64", "sint_jvp_f32",
                     "sint_precond_setup", "sint_precond_apply_f32", "sint_newton_solve"]:
        assert required in names


def test_library_exports_every_declared_symbol():
    from hpsint_b200 import _lib as L
    lib = L.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding gives every one a signature
    assert set(declared_functions()) <= set(L.SIGNATURES)


def test_create_rejects_bad_arguments_without_touching_the_gpu():
    from hpsint_b200 import _lib as L
    lib = L.lib()
    m = L.SintMesh()
    m.dim = 3
    for d in range(3):
        m.n_cells[d], m.h[d] = 4, 1.0
    p = L.SintParams(13, 16, 1, 1, 0.5, 1e-2, 1e-10, 4, 0.4, 1, 1)
    h = ctypes.c_void_p()
    assert lib.sint_create(ctypes.byref(m), ctypes.byref(p), ctypes.byref(h)) == 2  # SINT_ERR_GRAINS
    assert b"[1, 12]" in lib.sint_last_error()
    p.n_grains = 0
    assert lib.sint_create(ctypes.byref(m), ctypes.byref(p), ctypes.byref(h)) == 2
    p.n_grains = 4
    m.dim = 4
    assert lib.sint_create(ctypes.byref(m), ctypes.byref(p), ctypes.byref(h)) == 1  # SINT_ERR_ARG
    m.dim = 3
    m.h[1] = -1.0
    assert lib.sint_create(ctypes.byref(m), ctypes.byref(p), ctypes.byref(h)) == 1
    assert lib.sint_create(None, ctypes.byref(p), ctypes.byref(h)) == 1
    assert lib.sint_destroy(None) == 0
    assert lib.sint_newton_clear(None) == 1


def test_newton_defaults_mirror_hpsint():
    """lac/solvers_nonlinear_parameters.h:40-60"""
    from hpsint_b200 import _lib as L
    prm = L.SintNewtonParams()
    L.lib().sint_newton_default_params(ctypes.byref(prm))
    assert (prm.nl_max_iter, prm.nl_abs_tol, prm.nl_rel_tol) == (10, 1e-20, 1e-5)
    assert (prm.l_max_iter, prm.l_abs_tol, prm.l_rel_tol) == (1000, 1e-10, 1e-2)
    assert (prm.threshold_newton_iter, prm.threshold_linear_iter) == (100, 20)
    assert prm.use_damping == 1 and prm.reuse_preconditioner == 1 and prm.inner_precision == 64


def test_bdf_weights():
    """time_schemes.h:64-153"""
    from hpsint_b200 import bdf_weights
    dt = 0.1
    assert bdf_weights(1, [dt]) == pytest.approx([10.0, -10.0])
    assert bdf_weights(2, [dt, dt]) == pytest.approx([15.0, -20.0, 5.0])
    # effective order falls back to BDF1 before a second step exists
    assert bdf_weights(2, [dt, 0.0])[:2] == pytest.approx([10.0, -10.0])
    w = bdf_weights(3, [dt, dt, dt])
    assert w == pytest.approx([11 / 6 / dt, -3 / dt, 1.5 / dt, -1 / 3 / dt])
    assert sum(bdf_weights(2, [0.1, 0.3])) == pytest.approx(0.0, abs=1e-12)


def test_new_entry_points_reject_a_null_context():
    """Argument checks of the cut-off, tracker, periodic and advection entry
    points run before any device work (SINT_ERR_ARG = 1)."""
    from hpsint_b200 import _lib as L
    lib = L.lib()
    ok = ctypes.c_int()
    prm = L.SintAdvectionParams(1, 0, 1, 0, 1, 1)
    assert lib.sint_set_periodicity(None, 1) == 1
    assert lib.sint_distribute_constraints(None, None, None) == 1
    assert lib.sint_set_advection(None, None, None, 0, None) == 1
    assert lib.sint_set_advection_mechanism(None, None, None, 0, ctypes.byref(prm), None) == 1
    assert lib.sint_advection_forces(None, None, None, None) == 1
    assert lib.sint_advection_check_courant(None, 1.0, ctypes.byref(ok), None) == 1
    n = ctypes.c_int()
    assert lib.sint_grain_segment_periodicity(None, None, None, 0, ctypes.byref(n), None) == 1
    assert lib.sint_set_component_mask(None, None, 0.0, None) == 1
    assert lib.sint_set_cut_off_skip_zero_chunks(None, 1) == 1
