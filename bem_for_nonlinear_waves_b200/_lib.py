"""ctypes binding of the in-tree CUDA library (include/bem_b200.h).

The library is the product path: if it is missing this module raises, and the solver
API refuses to run without a CUDA device — there is no CPU fallback."""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libbem_b200.so")

c_int = ctypes.c_int32
c_dbl = ctypes.c_double
P_int = ctypes.POINTER(ctypes.c_int32)
P_dbl = ctypes.POINTER(ctypes.c_double)
P_u8 = ctypes.POINTER(ctypes.c_uint8)
P_i64 = ctypes.POINTER(ctypes.c_int64)

BEM_OK = 0
BEM_ERR_INVALID_ARGUMENT = -1
BEM_ERR_OUT_OF_MEMORY = -2
BEM_ERR_NOT_CONVERGED = -3
BEM_ERR_NAN = -4
BEM_ERR_DEVICE = -5
BEM_ERR_NOT_READY = -6
BEM_ERR_UNSUPPORTED = -7
STATUS = {0: "ok", -1: "invalid argument", -2: "out of memory", -3: "not converged", -4: "non-finite value",
          -5: "device error", -6: "not ready", -7: "unsupported"}


class Opts(ctypes.Structure):
    _fields_ = [("expansion_order", c_int), ("mac_theta", c_dbl), ("leaf_max_elements", c_int), ("max_level", c_int),
                ("tol", c_dbl), ("max_iter", c_int), ("device", c_int), ("tol_relative", c_int), ("preconditioner", c_int),
                ("precision", c_int), ("poly_degree", c_int), ("tree_on_host", c_int),
                ("tc_item_pairs", c_int), ("overlap_near", c_int), ("refine_rtol", c_dbl),
                ("tc_deterministic", c_int)]


class MelSurface(ctypes.Structure):
    _fields_ = [("n_points", c_int), ("X", P_dbl), ("n_faces", c_int), ("tri", P_int), ("face_dirichlet", P_u8),
                ("point_flags", P_u8), ("n_dof", c_int), ("face_dof", P_int), ("phi", P_dbl), ("phin", P_dbl)]


class Desc(ctypes.Structure):
    _fields_ = [("n_points", c_int), ("X", P_dbl), ("n_faces", c_int), ("tri", P_int), ("face_dirichlet", P_u8),
                ("n_dof", c_int), ("dof_point", P_int), ("dof_face", P_int), ("dof_kind", P_int), ("face_dof", P_int)]


class Stats(ctypes.Structure):
    _fields_ = [("iterations", c_int), ("converged", c_int), ("residual", c_dbl), ("residual_est", c_dbl),
                ("time_setup_s", c_dbl), ("time_solve_s", c_dbl), ("nnz_near", ctypes.c_int64), ("m2l_pairs", ctypes.c_int64),
                ("n_nodes", c_int), ("n_leaves", c_int), ("matvecs", c_int), ("matvecs_lo", c_int), ("time_device_s", c_dbl),
                ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
                ("time_plan_s", c_dbl), ("time_upload_s", c_dbl), ("time_setup_device_s", c_dbl), ("rhs_norm", c_dbl),
                ("tol_abs", c_dbl)]


EXPORTS = {
    "bem_gpu_is_available": (c_int, []),
    "bem_gpu_default_opts": (None, [ctypes.POINTER(Opts)]),
    "bem_gpu_create": (ctypes.c_void_p, [ctypes.POINTER(Opts)]),
    "bem_gpu_destroy": (None, [ctypes.c_void_p]),
    "bem_gpu_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "bem_gpu_build_dofs": (c_int, [c_int, P_dbl, c_int, P_int, P_u8, P_int, P_int, P_int, P_int, P_u8]),
    "bem_gpu_setup": (c_int, [ctypes.c_void_p, ctypes.POINTER(Desc)]),
    "bem_gpu_setup_refresh": (c_int, [ctypes.c_void_p, ctypes.POINTER(Desc)]),
    "bem_gpu_solve": (c_int, [ctypes.c_void_p, P_dbl, P_dbl, P_dbl, P_dbl, ctypes.POINTER(Stats)]),
    "bem_gpu_solve_bvp": (c_int, [ctypes.c_void_p, ctypes.POINTER(Desc), P_dbl, P_dbl, P_dbl, P_dbl, ctypes.POINTER(Stats)]),
    "bem_gpu_apply": (c_int, [ctypes.c_void_p, P_dbl, P_dbl, P_dbl]),
    "bem_gpu_point_integrals": (c_int, [ctypes.c_void_p, P_dbl, P_dbl, P_dbl, P_dbl]),
    "bem_gpu_matvec_device": (c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "bem_gpu_matvec_device_noalloc": (c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "bem_gpu_get_diag": (c_int, [ctypes.c_void_p, P_dbl]),
    "bem_gpu_scale_factor": (c_dbl, [ctypes.c_void_p]),
    "bem_gpu_near_row": (c_int, [ctypes.c_void_p, c_int, c_int, P_int, P_dbl, P_dbl]),
    "bem_gpu_face_leaf": (c_int, [ctypes.c_void_p, P_int, P_dbl]),
    "bem_gpu_tree_stats": (c_int, [ctypes.c_void_p, P_i64]),
    "bem_gpu_near_stats": (c_int, [ctypes.c_void_p, P_i64]),
    "bem_gpu_set_wait_limit": (c_int, [ctypes.c_void_p, ctypes.c_int64]),
    "bem_gpu_profile_matvec": (c_int, [ctypes.c_void_p, c_int, P_dbl]),
    "bem_gpu_matvec_device_mixed": (c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "bem_gpu_profile_matvec_mixed": (c_int, [ctypes.c_void_p, c_int, P_dbl]),
    "bem_gpu_check_device_status": (c_int, [ctypes.c_void_p]),
    "bem_gpu_fp64_peak_tflops": (c_dbl, [c_int]),
    "bem_gpu_poly_roots": (c_int, [ctypes.c_void_p, c_int, P_dbl, P_dbl]),
    "bem_gpu_setup_phases": (c_int, [ctypes.c_void_p, P_dbl]),
    "bem_gpu_tc_tuning": (c_int, [ctypes.c_void_p, P_int, P_int, P_dbl]),
    "bem_harmonic_ritz_values": (c_int, [c_int, P_dbl, c_int, P_dbl, P_dbl]),
    "bem_plan_inspect": (c_int, [ctypes.POINTER(Opts), ctypes.POINTER(Desc), P_int, P_dbl, P_i64]),
    "bem_plan_refresh_inspect": (c_int, [ctypes.POINTER(Opts), ctypes.POINTER(Desc), ctypes.POINTER(Desc), P_i64]),
    "bem_gpu_tree_check": (c_int, [ctypes.POINTER(Opts), ctypes.POINTER(Desc), P_i64]),
    "bem_gpu_mel_create": (ctypes.c_void_p, [c_int]),
    "bem_gpu_mel_destroy": (None, [ctypes.c_void_p]),
    "bem_gpu_mel_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "bem_gpu_mel_velocity": (c_int, [ctypes.c_void_p, ctypes.POINTER(MelSurface), P_dbl, P_dbl]),
    "bem_gpu_mel_stage": (c_int, [ctypes.c_void_p, ctypes.POINTER(MelSurface), c_int, c_dbl, c_dbl, P_dbl, P_dbl, P_dbl, P_dbl,
                                  P_dbl, P_dbl, P_dbl, P_dbl, P_dbl, P_dbl]),
    "bem_gpu_mel_phit_known": (c_int, [ctypes.c_void_p, ctypes.POINTER(MelSurface), P_int, P_int, P_int, P_int, c_int, P_dbl, c_dbl,
                                       P_dbl, P_dbl]),
    "bem_gpu_batch_create": (ctypes.c_void_p, [ctypes.POINTER(Opts), c_int]),
    "bem_gpu_batch_submit": (c_int, [ctypes.c_void_p, ctypes.POINTER(Desc), P_dbl, P_dbl, P_dbl, ctypes.POINTER(Stats),
                                     ctypes.POINTER(ctypes.c_int64)]),
    "bem_gpu_batch_poll": (c_int, [ctypes.c_void_p, ctypes.c_int64, c_int]),
    "bem_gpu_batch_release": (c_int, [ctypes.c_void_p, ctypes.c_int64]),
    "bem_gpu_batch_set_budget": (c_int, [ctypes.c_void_p, ctypes.c_int64]),
    "bem_gpu_batch_submit_chain": (c_int, [ctypes.c_void_p, ctypes.POINTER(Desc), P_u8, P_dbl, c_int, c_dbl, c_dbl, P_dbl, P_dbl,
                                           ctypes.POINTER(Stats), ctypes.POINTER(ctypes.c_int64)]),
    "bem_gpu_batch_stats": (c_int, [ctypes.c_void_p, P_i64]),
    "bem_gpu_device_bytes": (ctypes.c_int64, [ctypes.c_void_p]),
    "bem_gpu_estimate_bytes": (ctypes.c_int64, [ctypes.POINTER(Opts), ctypes.POINTER(Desc)]),
    "bem_gpu_batch_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "bem_gpu_batch_destroy": (None, [ctypes.c_void_p]),
}

_lib = None


def load():
    """Loads lib/libbem_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA library not built: {LIB_PATH} (run bem_for_nonlinear_waves_b200/build.py)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in EXPORTS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def ptr(a, t):
    return a.ctypes.data_as(t)
