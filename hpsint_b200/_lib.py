"""ctypes binding of libhpsint_b200.so (the C ABI in include/hpsint_b200.h).

The shared library is built in-tree by `make -C hpsint_b200/csrc`; there is
no fallback: importing the operator classes without it raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhpsint_b200.so")

MAX_GRAINS = 12

SINT_OK = 0
STATUS_NAMES = {
    0: "SINT_OK", 1: "SINT_ERR_ARG", 2: "SINT_ERR_GRAINS", 3: "SINT_ERR_CUDA",
    4: "SINT_ERR_NOT_READY", 5: "SINT_ERR_NO_CONVERGENCE", 6: "SINT_ERR_NEWTON",
    7: "SINT_ERR_NONFINITE", 8: "SINT_ERR_DT_MIN",
}

_c_int, _c_double, _c_void, _c_int64 = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_int64


class SintMesh(ctypes.Structure):
    _fields_ = [("dim", _c_int), ("n_cells", _c_int * 3), ("h", _c_double * 3), ("origin", _c_double * 3)]


class SintParams(ctypes.Structure):
    _fields_ = [("n_grains", _c_int), ("A", _c_double), ("B", _c_double), ("kappa_c", _c_double),
                ("kappa_p", _c_double), ("Mvol", _c_double), ("Mvap", _c_double), ("Msurf", _c_double),
                ("Mgb", _c_double), ("L", _c_double), ("tensorial", _c_int)]


class SintAdvectionParams(ctypes.Structure):
    _fields_ = [("k", _c_double), ("cgb", _c_double), ("ceq", _c_double), ("smoothening", _c_double),
                ("mt", _c_double), ("mr", _c_double)]


class SintResidualHooks(ctypes.Structure):
    _fields_ = [("perturb", _c_void), ("perturb_scale", _c_double), ("subtract", _c_void), ("scale", _c_double)]


class SintNewtonParams(ctypes.Structure):
    _fields_ = [("nl_max_iter", _c_int), ("nl_abs_tol", _c_double), ("nl_rel_tol", _c_double),
                ("l_max_iter", _c_int), ("l_abs_tol", _c_double), ("l_rel_tol", _c_double),
                ("gmres_restart", _c_int), ("threshold_newton_iter", _c_int),
                ("threshold_linear_iter", _c_int), ("use_damping", _c_int),
                ("reuse_preconditioner", _c_int), ("inner_precision", _c_int),
                ("right_preconditioning", _c_int)]


class SintNewtonStats(ctypes.Structure):
    _fields_ = [("newton_iterations", _c_int), ("linear_iterations", _c_int),
                ("residual_evaluations", _c_int), ("jacobian_setups", _c_int),
                ("preconditioner_setups", _c_int), ("initial_residual", _c_double),
                ("final_residual", _c_double)]


# name -> (restype, argtypes); every function declared in include/hpsint_b200.h
P = ctypes.POINTER
SIGNATURES = {
    "sint_create": (_c_int, [P(SintMesh), P(SintParams), P(_c_void)]),
    "sint_destroy": (_c_int, [_c_void]),
    "sint_dof_layout": (_c_int, [_c_void, P(_c_int64), P(_c_int), P(_c_int64)]),
    "sint_set_time_weights": (_c_int, [_c_void, _c_double, P(_c_double), _c_int, _c_double]),
    "sint_set_mobility": (_c_int, [_c_void, _c_double, _c_double, _c_double, _c_double, _c_double]),
    "sint_set_linearization_point": (_c_int, [_c_void, _c_void, _c_void]),
    "sint_residual_f64": (_c_int, [_c_void, _c_void, _c_void, P(_c_void), _c_int, _c_void]),
    "sint_residual_f64_hooks": (_c_int, [_c_void, _c_void, _c_void, P(_c_void), _c_int, P(SintResidualHooks),
                                         _c_void]),
    "sint_jvp_f64": (_c_int, [_c_void, _c_void, _c_void, _c_void]),
    "sint_jvp_f32": (_c_int, [_c_void, _c_void, _c_void, _c_void]),
    "sint_jvp_f64_noalloc": (_c_int, [P(SintMesh), P(SintParams), _c_double, _c_double, _c_void, _c_void, _c_void,
                                      _c_void]),
    "sint_precond_setup": (_c_int, [_c_void, _c_void]),
    "sint_precond_apply_f64": (_c_int, [_c_void, _c_void, _c_void, _c_void]),
    "sint_precond_apply_f32": (_c_int, [_c_void, _c_void, _c_void, _c_void]),
    "sint_ac_inverse_diagonal_f64": (_c_int, [_c_void, _c_void, _c_void]),
    "sint_set_preconditioner_type": (_c_int, [_c_void, _c_int]),
    "sint_ch_matrix_f64": (_c_int, [_c_void, _c_void, _c_void]),
    "sint_ch_blocks_f64": (_c_int, [_c_void, _c_void, _c_void]),
    "sint_set_component_mask": (_c_int, [_c_void, _c_void, _c_double, _c_void]),
    "sint_component_mask_statistics": (_c_int, [_c_void, P(_c_int64), _c_void]),
    "sint_set_preconditioner_cut_off": (_c_int, [_c_void, _c_int]),
    "sint_set_cut_off_skip_zero_chunks": (_c_int, [_c_void, _c_int]),
    "sint_cut_off_freeze": (_c_int, [_c_void, _c_void, _c_void, _c_void]),
    "sint_grain_segments": (_c_int, [_c_void, _c_void, _c_double, _c_void, P(_c_int), _c_void]),
    "sint_grain_segment_properties": (_c_int, [_c_void, _c_void, _c_void, _c_int, P(_c_double), _c_void]),
    "sint_get_component_mask": (_c_int, [_c_void, _c_void, _c_void]),
    "sint_grain_segment_periodicity": (_c_int, [_c_void, _c_void, P(_c_int), _c_int, P(_c_int), _c_void]),
    "sint_set_periodicity": (_c_int, [_c_void, ctypes.c_uint]),
    "sint_distribute_constraints": (_c_int, [_c_void, _c_void, _c_void]),
    "sint_set_advection": (_c_int, [_c_void, _c_void, _c_void, _c_int, _c_void]),
    "sint_set_advection_mechanism": (_c_int, [_c_void, _c_void, _c_void, _c_int, P(SintAdvectionParams), _c_void]),
    "sint_advection_forces": (_c_int, [_c_void, _c_void, _c_void, _c_void]),
    "sint_advection_check_courant": (_c_int, [_c_void, _c_double, P(_c_int), _c_void]),
    "sint_vec_axpy_f64": (_c_int, [_c_int64, _c_double, _c_void, _c_void, _c_void]),
    "sint_vec_sadd_f64": (_c_int, [_c_int64, _c_double, _c_double, _c_void, _c_void, _c_void]),
    "sint_vec_scale_f64": (_c_int, [_c_int64, _c_double, _c_void, _c_void]),
    "sint_vec_dot_f64": (_c_int, [_c_void, _c_int64, _c_void, _c_void, _c_void, _c_void]),
    "sint_vec_norm2_f64": (_c_int, [_c_void, _c_int64, _c_void, _c_void, _c_void]),
    "sint_vec_axpy_f32": (_c_int, [_c_int64, ctypes.c_float, _c_void, _c_void, _c_void]),
    "sint_vec_dot_f32": (_c_int, [_c_void, _c_int64, _c_void, _c_void, _c_void, _c_void]),
    "sint_vec_norm2_f32": (_c_int, [_c_void, _c_int64, _c_void, _c_void, _c_void]),
    "sint_vec_f64_to_f32": (_c_int, [_c_int64, _c_void, _c_void, _c_void]),
    "sint_vec_f32_to_f64": (_c_int, [_c_int64, _c_void, _c_void, _c_void]),
    "sint_vec_select_f64": (_c_int, [_c_int64, _c_void, _c_void, _c_void, _c_void, _c_void, _c_void]),
    "sint_newton_default_params": (None, [P(SintNewtonParams)]),
    "sint_newton_clear": (_c_int, [_c_void]),
    "sint_newton_solve": (_c_int, [_c_void, _c_void, P(_c_void), P(SintNewtonParams), P(SintNewtonStats),
                                   _c_void]),
    "sint_nn_conv3x3_f32": (_c_int, [_c_void, _c_int, _c_int, _c_int, _c_int, _c_void, _c_void, _c_void, _c_int,
                                     _c_int, _c_void]),
    "sint_nn_conv3x3_flip_f32": (_c_int, [_c_void, _c_int, _c_int, _c_void, _c_void]),
    "sint_nn_conv3x3_wgrad_workspace": (_c_int64, [_c_int, _c_int, _c_int, _c_int, _c_int]),
    "sint_nn_conv3x3_wgrad_f32": (_c_int, [_c_void, _c_void, _c_int, _c_int, _c_int, _c_int, _c_int, _c_void, _c_void,
                                           _c_int, _c_void, _c_void]),
    "sint_nn_leaky_relu_f32": (_c_int, [_c_int64, ctypes.c_float, _c_void, _c_void, _c_void]),
    "sint_nn_leaky_relu_bwd_f32": (_c_int, [_c_int64, ctypes.c_float, _c_void, _c_void, _c_void, _c_void]),
    "sint_nn_grain_sum_f32": (_c_int, [_c_void, _c_int, _c_int, _c_int64, _c_void, _c_void]),
    "sint_nn_grain_bcast_add_f32": (_c_int, [_c_void, _c_int, _c_int, _c_int64, _c_void, _c_void]),
    "sint_nn_adam_f32": (_c_int, [_c_int64, _c_void, _c_void, _c_void, _c_void, ctypes.c_float, ctypes.c_float,
                                  ctypes.c_float, ctypes.c_float, _c_int, _c_void]),
    "sint_nn_mse_workspace": (_c_int64, []),
    "sint_nn_mse_f32": (_c_int, [_c_int64, _c_void, _c_void, _c_void, _c_void, _c_void, _c_void, _c_void]),
    "sint_nn_features_f64": (_c_int, [_c_void, _c_void, _c_int64, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int,
                                      _c_int, ctypes.c_float, _c_void, _c_void, _c_void, _c_int, _c_void]),
    "sint_nn_targets_f64": (_c_int, [_c_void, _c_void, _c_void, _c_int64, _c_int, _c_int, _c_int, _c_int, _c_int,
                                     _c_int, _c_int, ctypes.c_float, _c_void, _c_void, _c_void, _c_int, _c_void]),
    "sint_nn_conv3x3_tc_f32": (_c_int, [_c_void, _c_int, _c_int, _c_int, _c_int, _c_void, _c_void, _c_void, _c_int,
                                        _c_int, _c_void, _c_void]),
    "sint_nn_conv3x3_tc_ex_f32": (_c_int, [_c_void, _c_int, _c_int, _c_int, _c_int, _c_void, _c_void, _c_void,
                                           _c_int, _c_int, _c_void, _c_int, _c_int, ctypes.c_float, _c_void,
                                           _c_void]),
    "sint_nn_weighted_diff_f32": (_c_int, [_c_int64, _c_void, _c_void, _c_void, _c_void, _c_void]),
    "sint_nn_mul_add_f32": (_c_int, [_c_int64, ctypes.c_float, _c_void, _c_void, _c_void, _c_void]),
    "sint_nn_increment_scales_f64": (_c_int, [_c_void, _c_void, _c_int64, _c_int64, _c_int, ctypes.c_float,
                                              ctypes.c_float, _c_void, _c_void, _c_void, _c_void, _c_void]),
    "sint_nn_apply_guess_f64": (_c_int, [_c_void, _c_void, _c_int64, _c_int64, _c_int, ctypes.c_float, _c_void,
                                         _c_void, _c_void, _c_void, _c_void]),
    "sint_nn_features3d_f64": (_c_int, [_c_void, _c_void, _c_int64] + [_c_int] * 10 +
                               [ctypes.c_float, _c_void, _c_void, _c_void, _c_int, _c_void]),
    "sint_nn_targets3d_f64": (_c_int, [_c_void, _c_void, _c_void, _c_int64] + [_c_int] * 10 +
                              [ctypes.c_float, _c_void, _c_void, _c_void, _c_int, _c_void]),
    "sint_nn_apply_guess3d_f64": (_c_int, [_c_void, _c_void, _c_int64] + [_c_int] * 7 +
                                  [ctypes.c_float, _c_void, _c_void, _c_void, _c_void, _c_void]),
    "sint_nn_zero_pad_slices_f32": (_c_int, [_c_void, _c_int, _c_int, _c_int64, _c_void]),
    "sint_nn_conv3d_f32": (_c_int, [_c_int] * 4 + [_c_void, _c_int, _c_void, _c_void, _c_int, _c_void, _c_void, _c_void,
                                                    _c_int, _c_int, ctypes.c_float, _c_void, _c_int, _c_int, _c_void]),
    "sint_last_error": (ctypes.c_char_p, []),
    "sint_kernel_launch_count": (_c_int64, []),
}

_lib = None


class SintError(RuntimeError):
    def __init__(self, status, where, message):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{where}: {self.status_name}: {message}")


def lib():
    """Load the in-tree library; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not found: build it with `make -C hpsint_b200/csrc` "
                              "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error():
    """Text of the last error the library recorded on this thread."""
    return lib().sint_last_error().decode(errors="replace")


def check(status, where):
    if status != SINT_OK:
        msg = lib().sint_last_error().decode(errors="replace")
        raise SintError(status, where, msg)


def kernel_launch_count():
    return int(lib().sint_kernel_launch_count())
