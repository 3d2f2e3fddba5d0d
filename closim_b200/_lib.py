"""ctypes binding of libclosim_cuda.so (the C ABI declared in include/closim_cuda.h).

The library is built in-tree by closim_b200/csrc/Makefile. Loading fails loudly
when it is missing: there is no CPU fallback.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libclosim_cuda.so")

CS_OK, CS_E_UNINIT, CS_E_NONFINITE, CS_E_CAPACITY, CS_E_CUDA, CS_E_ARG = range(6)
CS_PRECISION_FP64, CS_PRECISION_MIXED = 0, 1
CS_PRECOND_JACOBI, CS_PRECOND_SCHWARZ, CS_PRECOND_MAS2 = 0, 1, 2
CS_BROADPHASE_MIRROR, CS_BROADPHASE_EXACT = 0, 1


class cs_material(C.Structure):
    _fields_ = [(k, C.c_double) for k in ["areal_density", "thickness", "stretch_warp", "stretch_weft",
                                           "stretch_coupling", "shear", "bend_warp", "bend_weft", "damping"]]


class cs_contact_params(C.Structure):
    _fields_ = [(k, C.c_double) for k in ["dhat", "kappa", "dmin", "mu", "eps"]]


class cs_mesh(C.Structure):
    _fields_ = [("n", C.c_int32), ("m", C.c_int32), ("hg", C.c_int32), ("indices", C.c_void_p),
                ("rest", C.c_void_p), ("inv_dm", C.c_void_p), ("area", C.c_void_p), ("mass", C.c_void_p),
                ("hinge", C.c_void_p), ("hinge_meta", C.c_void_p)]


class cs_stepper_options(C.Structure):
    _fields_ = [("newton_iters", C.c_int32), ("pcg_max_iters", C.c_int32), ("ls_iters", C.c_int32),
                ("precond", C.c_int32), ("grad_tol", C.c_double)]


class cs_step_stats(C.Structure):
    _fields_ = [("newton_iters", C.c_int32), ("pcg_iters", C.c_int32), ("grad_norm", C.c_double),
                ("energy", C.c_double), ("max_strain", C.c_double), ("converged", C.c_int32),
                ("has_contact", C.c_int32)] + \
               [(k, C.c_double) for k in ["candidate_pairs", "active_pairs", "vt_pairs", "ee_pairs", "floor_pairs",
                                          "min_distance", "min_toi", "barrier_energy", "friction_work",
                                          "rejected_line_search_steps", "ccd_failures"]] + \
               [("newton_iters_used", C.c_int32), ("armijo_trials", C.c_int32)]


class cs_broadphase_diag(C.Structure):
    _fields_ = [("scanned_count", C.c_int64), ("written_count", C.c_int64), ("capacity", C.c_int64),
                ("candidate_overflow", C.c_int32), ("tree_depth", C.c_int32), ("root", C.c_int32),
                ("reserved", C.c_int32)]


EXPORTS = ["cs_create", "cs_destroy", "cs_last_error", "cs_initialize", "cs_set_contact",
           "cs_set_stepper_options", "cs_set_material", "cs_set_pins", "cs_step", "cs_get_positions",
           "cs_get_velocities", "cs_set_state", "cs_last_stats", "cs_membrane_hvp", "cs_step_n", "cs_sync",
           "cs_kernel_launches", "cs_stream", "cs_profile", "cs_profile_read", "cs_profile_phases", "cs_solver_info", "cs_forward", "cs_backward",
           "cs_set_adjoint_options", "cs_adjoint_stats", "cs_set_newton_mode", "cs_batch_create", "cs_batch_destroy",
           "cs_batch_last_error", "cs_batch_initialize", "cs_batch_set_contact", "cs_batch_set_stepper_options",
           "cs_batch_step", "cs_batch_get_positions", "cs_batch_get_velocities", "cs_batch_stats",
           "cs_batch_autotune", "cs_batch_set_threads", "cs_batch_stream", "cs_batch_launch_shape", "cs_session_step", "cs_session_reset",
           "cs_session_restore_stable", "cs_build_grid",
           "cs_preprocess", "cs_contact_active", "cs_update_static_positions", "cs_set_graph_mode", "cs_graph_info", "cs_internal_energy", "cs_internal_gradient", "cs_membrane_hvp_analytic",
           "cs_broadphase_create", "cs_broadphase_destroy", "cs_broadphase_last_error",
           "cs_broadphase_build", "cs_broadphase_diagnostics", "cs_broadphase_pairs", "cs_broadphase_state"]

_lib = None


def load():
    """Load the CUDA solver library (raises OSError if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with `make -C closim_b200/csrc` "
                      "(the CUDA solver has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "cs_create": (vp, [C.c_int, C.c_int]),
        "cs_destroy": (None, [vp]),
        "cs_last_error": (C.c_char_p, [vp]),
        "cs_initialize": (C.c_int, [vp, C.POINTER(cs_mesh), C.POINTER(cs_material), vp, vp, vp]),
        "cs_set_contact": (C.c_int, [vp, C.POINTER(cs_contact_params), C.c_int, C.c_double, vp, C.c_int32, vp,
                                     C.c_int32]),
        "cs_set_stepper_options": (C.c_int, [vp, C.POINTER(cs_stepper_options)]),
        "cs_set_material": (C.c_int, [vp, C.POINTER(cs_material)]),
        "cs_set_pins": (C.c_int, [vp, C.c_int32, vp, vp]),
        "cs_step": (C.c_int, [vp, C.c_double]),
        "cs_step_n": (C.c_int, [vp, C.c_double, C.c_int32]),
        "cs_get_positions": (C.c_int, [vp, vp]),
        "cs_get_velocities": (C.c_int, [vp, vp]),
        "cs_set_state": (C.c_int, [vp, vp, vp]),
        "cs_last_stats": (C.c_int, [vp, C.POINTER(cs_step_stats)]),
        "cs_membrane_hvp": (C.c_int, [vp, vp, vp, vp]),
        "cs_internal_energy": (C.c_int, [vp, vp, vp]),
        "cs_contact_active": (C.c_int, [vp, C.c_int32, vp, vp, vp]),
        "cs_set_graph_mode": (C.c_int, [vp, C.c_int32]),
        "cs_update_static_positions": (C.c_int, [vp, vp, C.c_int32]),
        "cs_graph_info": (C.c_int, [vp, vp]),
        "cs_internal_gradient": (C.c_int, [vp, vp, vp, vp, vp]),
        "cs_membrane_hvp_analytic": (C.c_int, [vp, vp, vp, vp]),
        "cs_sync": (C.c_int, [vp]),
        "cs_kernel_launches": (C.c_int64, [vp]),
        "cs_stream": (vp, [vp]),
        "cs_profile": (C.c_int, [vp, C.c_int]),
        "cs_profile_read": (C.c_int, [vp, vp]),
        "cs_profile_phases": (C.c_int, [vp, vp, C.c_int32]),
        "cs_solver_info": (C.c_int, [vp, vp, C.c_int32]),
        "cs_forward": (C.c_int, [vp, C.c_double, C.c_int32, C.c_int32]),
        "cs_backward": (C.c_int, [vp, vp, vp, vp]),
        "cs_set_adjoint_options": (C.c_int, [vp, C.c_int32, C.c_double]),
        "cs_adjoint_stats": (C.c_int, [vp, vp]),
        "cs_set_newton_mode": (C.c_int, [vp, C.c_int32, C.c_double]),
        "cs_batch_create": (vp, [C.c_int32]),
        "cs_batch_destroy": (None, [vp]),
        "cs_batch_last_error": (C.c_char_p, [vp]),
        "cs_batch_initialize": (C.c_int, [vp, C.c_int32, vp, vp, vp, vp, vp, vp, vp, vp]),
        "cs_batch_set_contact": (C.c_int, [vp, C.POINTER(cs_contact_params), C.c_int32, C.c_double]),
        "cs_batch_set_stepper_options": (C.c_int, [vp, C.POINTER(cs_stepper_options)]),
        "cs_batch_step": (C.c_int, [vp, C.c_double, C.c_int32]),
        "cs_batch_get_positions": (C.c_int, [vp, vp]),
        "cs_batch_get_velocities": (C.c_int, [vp, vp]),
        "cs_batch_stats": (C.c_int, [vp, vp]),
        "cs_batch_autotune": (C.c_int, [vp, C.c_double, C.POINTER(C.c_int32)]),
        "cs_batch_set_threads": (C.c_int, [vp, C.c_int32]),
        "cs_batch_stream": (vp, [vp]),
        "cs_batch_launch_shape": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
        "cs_session_step": (C.c_int, [vp, C.c_double, vp, C.POINTER(C.c_int32)]),
        "cs_session_reset": (C.c_int, [vp]),
        "cs_session_restore_stable": (C.c_int, [vp, C.POINTER(C.c_int32)]),
        "cs_build_grid": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, vp, vp, vp]),
        "cs_preprocess": (C.c_int, [C.c_int32, C.c_int32, vp, vp, vp, C.c_double, vp, vp, vp,
                                    C.POINTER(C.c_int32), vp, vp]),
        "cs_broadphase_create": (vp, [C.c_int32, C.c_int32, vp, C.c_double, C.c_int64, C.c_int32]),
        "cs_broadphase_destroy": (None, [vp]),
        "cs_broadphase_last_error": (C.c_char_p, [vp]),
        "cs_broadphase_build": (C.c_int, [vp, vp, vp]),
        "cs_broadphase_diagnostics": (C.c_int, [vp, C.POINTER(cs_broadphase_diag)]),
        "cs_broadphase_pairs": (C.c_int, [vp, vp]),
        "cs_broadphase_state": (C.c_int, [vp] + [vp] * 9),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
