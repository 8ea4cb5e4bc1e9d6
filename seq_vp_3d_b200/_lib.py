"""ctypes binding of libsvp3d.so (the sm_100a CUDA library built from seq_vp_3d_b200/csrc).

There is no CPU fallback: if the library is missing or CUDA is unavailable, every entry point raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsvp3d.so")

P, I64, D, I32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int32

SVP_OK, SVP_EINVAL, SVP_ECUDA, SVP_ENOMEM, SVP_ENUMERIC = 0, 1, 2, 3, 4


class SvpError(RuntimeError):
    """A libsvp3d call returned a non-zero status."""

    def __init__(self, code, message):
        super().__init__(f"libsvp3d error {code}: {message}")
        self.code = code


class Grid(ctypes.Structure):
    _fields_ = [("nx", I64), ("ny", I64), ("nz", I64), ("hx", D), ("hy", D), ("hz", D),
                ("x0", D), ("y0", D), ("z0", D)]


class CertConfig(ctypes.Structure):
    _fields_ = [("delta", D), ("max_depth", I64), ("max_boxes", I64), ("tile_size", I64),
                ("prescreen", I32), ("execution", I32)]


class CertResult(ctypes.Structure):
    _fields_ = [("status", I32), ("reason", I32), ("n_cells_checked", I64), ("n_uncertain", I64),
                ("n_infeasible", I64), ("n_boxes", I64), ("max_depth", I64), ("witness_cell", I64),
                ("n_fast_cells", I64), ("n_fallback_cells", I64), ("n_prescreen_cells", I64),
                ("has_min_jd", I32), ("has_sampled_min", I32), ("min_jd_lower_bound", D),
                ("min_margin_lower_bound", D), ("sampled_min_jd", D), ("witness_point", D * 3)]


class CellVerdict(ctypes.Structure):
    _fields_ = [("status", I32), ("reason", I32), ("has_margin", I32), ("has_witness", I32),
                ("boxes", I64), ("depth", I64), ("margin", D), ("witness", D * 3)]


class Weights(ctypes.Structure):
    _fields_ = [("lam", D), ("mu", D), ("nu", D), ("kappa", D), ("activation", D), ("delta", D)]


class PreParams(ctypes.Structure):
    _fields_ = [(n, D) for n in ("mu", "alpha", "kappa", "j0", "lr", "cap", "sigma_grad", "sigma_field", "beta1",
                                 "beta2", "eps")]


# name -> argtypes (restype int)
SIGNATURES = {
    "svp_last_error": [ctypes.c_char_p, ctypes.c_size_t],
    "svp_version": [],
    "svp_counters": [P],
    "svp_timers_enable": [ctypes.c_int],
    "svp_timer_read": [ctypes.c_char_p, P, P],
    "svp_edge_hull_margins": [P, P, D, P, P, P],
    "svp_edge_hull_margins_directed": [P, P, D, P, P, P],
    "svp_prescreen_lower_bounds": [P, P, P, I64, P, P],
    "svp_fallback_arrays": [P, I64, P, D, P, P, P, P, P, P, P],
    "svp_fallback_arrays_directed": [P, I64, P, D, P, P, P, P, P, P, P],
    "svp_classify_cells": [P, P, P, P, I64, D, I64, I64, P, P],
    "svp_classify_cells_noalloc": [P, P, P, P, I64, D, I64, I64, P, P],
    "svp_classify_cells_policy": [P, P, P, P, I64, D, I64, I64, I32, P, P],
    "svp_certifier_create": [P, P, P],
    "svp_certifier_destroy": [P],
    "svp_certify_map": [P, P, P, P],
    "svp_pair_create": [P, P, P, P, P, P, P],
    "svp_pair_set_reference": [P, P, P],
    "svp_pair_destroy": [P],
    "svp_pair_spline_coefficients": [P, P, P],
    "svp_pair_set_spline_coefficients": [P, P, P],
    "svp_warp": [P, P, P, P, P],
    "svp_sample_points": [P, P, I64, P, P, P],
    "svp_energy": [P, P, P, P, P, P],
    "svp_energy_difference": [P, P, P, P, P, P, P],
    "svp_trial_energy": [P, P, P, P, P, P, P, P, P, P],
    "svp_trial_energy_masked": [P, P, P, P, P, P, P, P, P, P, P],
    "svp_trial_energy_active": [P, P, P, P, P, P, P, P, P, P, P, P],
    "svp_trial_energy_screened": [P, P, P, P, P, P, P, P, P, P, P, P, P],
    "svp_gradient_masked": [P, P, P, P, ctypes.c_int32, P, P, P],
    "svp_outer_gradients_masked": [P, P, P, P, P, P, P, P, P],
    "svp_ggn_diagonal_masked": [P, P, P, P, P, P],
    "svp_energy_difference_masked": [P, P, P, P, P, P, P, P, P],
    "svp_energy_difference_screened": [P, P, P, P, P, P, P, P, P],
    "svp_pair_set_precision": [P, ctypes.c_int32],
    "svp_dot_dev": [P, P, I64, P, P],
    "svp_bb2_dots_dev": [P, P, P, P, P, P, I64, P, P],
    "svp_max_abs_diff_dev": [P, P, I64, P, P],
    "svp_step_bound_dev": [P, P, P, P, P],
    "svp_trial_point": [P, P, D, P, P, P, P, P],
    "svp_step_dots_dev": [P, P, P, P, P, P, I64, P, P],
    "svp_pre_energy_grad": [P, P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, D, D, D, P, D, D, D, D, P, P, P],
    "svp_pre_level": [P, P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, D, D, D, P, ctypes.c_int32, ctypes.c_int32,
                      P, P, P, P, P, P, P],
    "svp_image_downsample": [P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, P, ctypes.c_int32, ctypes.c_int32,
                             ctypes.c_int32, P],
    "svp_field_prolong": [P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, P, ctypes.c_int32, ctypes.c_int32,
                          ctypes.c_int32, P, P, P],
    "svp_gradient": [P, P, P, P, I32, P, P],
    "svp_outer_gradients": [P, P, P, P, P, P, P, P],
    "svp_ggn_diagonal": [P, P, P, P, P],
    "svp_ggn_hvp": [P, P, P, P, P, P],
    "svp_node_min_jd": [P, P, P, P],
    "svp_node_min_jd_extended": [P, P, ctypes.c_double, P, P, P],
    "svp_jd_root": [P, P, P, D, P, P, P],
    "svp_poisson_apply": [P, D, D, I32, P, P, D, P, P],
    "svp_dot": [P, P, I64, P, P],
    "svp_axpy": [P, D, P, I64, P, P],
    "svp_inject": [P, P, P, P],
    "svp_restrict": [P, P, P, P],
    "svp_step_bound": [P, P, P, P, P],
    "svp_bb2_dots": [P, P, P, P, P, P, I64, P, P],
    "svp_max_abs_diff": [P, P, I64, P, P],
    "svp_image_shift": [P, P, D, P, P],
    "svp_pg_scale": [P, P, P, D, D, D, P, P, P],
}

TERM_IMAGE, TERM_PROXIMITY, TERM_JD, TERM_CURL, TERM_BARRIER = 1, 2, 4, 8, 16
TERMS = {"image": 1, "proximity": 2, "jd": 4, "curl": 8, "barrier": 16, "total": 31, "outer": 17}

_lib = None


def load():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m seq_vp_3d_b200.build` (no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        _lib = lib
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(4096)
    load().svp_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(code):
    if code != SVP_OK:
        raise SvpError(code, last_error())
    return code


def call(name, *args):
    return check(getattr(load(), name)(*args))
