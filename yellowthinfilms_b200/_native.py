"""ctypes binding of libytf.so (the C ABI of include/ytf.h).

There is no CPU fallback: if the library is missing or no CUDA device is present the
calls raise. Build it with ``python -m yellowthinfilms_b200.build``.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libytf.so")

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)
_u8 = ctypes.POINTER(ctypes.c_ubyte)
_vp = ctypes.c_void_p

class TransferDesc(ctypes.Structure):
    """ytf_transfer_desc (include/ytf.h)."""
    # array fields as raw addresses (ints): the same C ABI as typed pointers, filled without a
    # ctypes cast per field
    _fields_ = [("stack", _vp), ("omega", ctypes.c_double), ("source_layer", ctypes.c_int), ("nk", ctypes.c_int),
                ("k_nodes", _vp), ("k_weights", _vp), ("nphi", ctypes.c_int), ("phi_nodes", _vp), ("phi_weights", _vp),
                ("nobs", ctypes.c_int), ("obs_layers", _vp), ("check_symmetry", ctypes.c_int),
                ("rotation", ctypes.c_int), ("is2d", ctypes.c_int), ("nodes_on_device", ctypes.c_int)]


class GreenDesc(ctypes.Structure):
    """ytf_green_desc (include/ytf.h)."""
    _fields_ = [("cache", _vp), ("obs_layer", ctypes.c_int), ("zsrc_local", ctypes.c_double), ("nz", ctypes.c_int),
                ("z_obs", _vp), ("nx", ctypes.c_int), ("xs", _vp), ("ny", ctypes.c_int), ("ys", _vp),
                ("terms", ctypes.c_int), ("precision", ctypes.c_int), ("out", _vp), ("out_is_device", ctypes.c_int)]


class Tune(ctypes.Structure):
    """ytf_tune (include/ytf.h)."""
    _fields_ = [("block", ctypes.c_int), ("ctas_per_sm", ctypes.c_int), ("tile", ctypes.c_int), ("chunk", ctypes.c_int),
                ("synth_ctas_per_sm", ctypes.c_int)]


class GridParams(ctypes.Structure):
    """ytf_grid_params (include/ytf.h)."""
    _fields_ = [("h_min", ctypes.c_double), ("rho_max", ctypes.c_double), ("target_decay", ctypes.c_double),
                ("kr_cap", ctypes.c_double), ("scan", ctypes.c_int), ("order", ctypes.c_int), ("rtol", ctypes.c_double)]


class GridInfo(ctypes.Structure):
    """ytf_grid_info (include/ytf.h)."""
    _fields_ = [("Kcut", ctypes.c_double), ("kmax", ctypes.c_double), ("n_panels", ctypes.c_long),
                ("n_poles", ctypes.c_int), ("n_light_lines", ctypes.c_int), ("poles", (ctypes.c_double * 2) * 256),
                ("light_lines", ctypes.c_double * 64), ("panels", _d), ("panels_cap", ctypes.c_long)]


# name -> (restype, argtypes); every symbol include/ytf.h declares
SIGNATURES = {
    "ytf_version": (ctypes.c_int, []),
    "ytf_ctx_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int]),
    "ytf_ctx_destroy": (ctypes.c_int, [_vp]),
    "ytf_ctx_set_stream": (ctypes.c_int, [_vp, _vp]),
    "ytf_ctx_set_wait_limit": (ctypes.c_int, [_vp, ctypes.c_long]),
    "ytf_ctx_set_group_bytes": (ctypes.c_int, [_vp, ctypes.c_long]),
    "ytf_ctx_sync": (ctypes.c_int, [_vp]),
    "ytf_last_error": (ctypes.c_char_p, [_vp]),
    "ytf_ctx_profile": (ctypes.c_int, [_vp, ctypes.c_int]),
    "ytf_ctx_profile_read": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_char_p, _d, ctypes.POINTER(ctypes.c_long), _i]),
    "ytf_stack_create": (ctypes.c_int, [_vp, ctypes.c_int, _i, _i, _d, _d, _d, ctypes.POINTER(_vp)]),
    "ytf_stack_destroy": (ctypes.c_int, [_vp]),
    "ytf_transfer_1d": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, _d, _d, ctypes.c_int, _i,
                                       ctypes.c_int, ctypes.POINTER(_vp)]),
    "ytf_transfer_2d": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, _d, _d, ctypes.c_int, _d, _d,
                                       ctypes.c_int, _i, ctypes.c_int, ctypes.POINTER(_vp)]),
    "ytf_cache_destroy": (ctypes.c_int, [_vp]),
    "ytf_cache_info": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_long), _i, _i, _i, _i]),
    "ytf_cache_status": (ctypes.c_int, [_vp, _vp, _u8, _u8, _u8]),
    "ytf_cache_export": (ctypes.c_int, [_vp, _vp, _d, _d, _d, _d, _d, _d]),
    "ytf_green": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, _d, ctypes.c_int, _d, ctypes.c_int,
                                 _d, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int]),
    "ytf_green_noalloc": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                         ctypes.c_int, _vp, ctypes.c_int, _vp]),
    "ytf_cavity_response": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.c_long, _d, ctypes.c_double,
                                           _d]),
    "ytf_cavity_response_batch": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp), _d, _i,
                                                 ctypes.POINTER(ctypes.c_long), _d, ctypes.c_double, _d]),
    "ytf_gl_rule_batch": (ctypes.c_int, [_vp, ctypes.c_int, _i, _d, _d, ctypes.c_int, _i, _d, _d, _d]),
    "ytf_rule_panels_batch": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp), _d, _i, ctypes.POINTER(GridParams),
                                             _i, _d, _d, ctypes.c_long, _d, ctypes.POINTER(ctypes.c_long),
                                             ctypes.POINTER(ctypes.c_long)]),
    "ytf_gl_rule_batch_device": (ctypes.c_int, [_vp, ctypes.c_int, _i, _d, _d, ctypes.c_int, _i, _d, _vp, _vp]),
    "ytf_layer_light_lines": (ctypes.c_int, [_d, _d, ctypes.c_double, ctypes.c_double, _d, _i]),
    "ytf_nodes_1d": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(GridParams), ctypes.c_long, _d,
                                    _d, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(GridInfo)]),
    "ytf_mlp_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _i, ctypes.c_ulonglong, ctypes.POINTER(_vp)]),
    "ytf_mlp_destroy": (ctypes.c_int, [_vp]),
    "ytf_mlp_last_error": (ctypes.c_char_p, [_vp]),
    "ytf_mlp_num_params": (ctypes.c_long, [_vp]),
    "ytf_mlp_set_stream": (ctypes.c_int, [_vp, _vp]),
    "ytf_mlp_params": (ctypes.c_int, [_vp, _vp, _vp]),
    "ytf_mlp_forward": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int]),
    "ytf_mlp_gradients": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_float),
                                         ctypes.c_int]),
    "ytf_mlp_train": (ctypes.c_int, [_vp, ctypes.c_long, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                     ctypes.c_ulonglong, _vp]),
    "ytf_peaks_batch": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _d, _d, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_long, _i, _d, _d, ctypes.POINTER(ctypes.c_long)]),
    "ytf_adaptive_seeds": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(GridParams),
                                          ctypes.c_long, _d, ctypes.POINTER(ctypes.c_long)]),
    "ytf_nodes_2d": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(GridParams), ctypes.c_int,
                                    ctypes.c_long, _d, _d, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long),
                                    ctypes.POINTER(GridInfo)]),
    "ytf_nodes_from_poles": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(GridParams),
                                            ctypes.c_int, _d, _d, ctypes.c_long, _d, _d, ctypes.POINTER(ctypes.c_long),
                                            ctypes.POINTER(GridInfo)]),
    "ytf_transfer_1d_contour": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, _d, _d, _d, _d,
                                               ctypes.c_int, _i, ctypes.POINTER(_vp)]),
    "ytf_bessel_j01": (ctypes.c_int, [_vp, ctypes.c_long, _d, _d, _d]),
    "ytf_bessel_j": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_long, _d, _d, _d, _d]),
    "ytf_transfer_batch": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(TransferDesc), ctypes.POINTER(_vp)]),
    "ytf_green_batch": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(GreenDesc)]),
    "ytf_plan_create": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(TransferDesc), ctypes.POINTER(GreenDesc),
                                       ctypes.POINTER(Tune), ctypes.POINTER(_vp)]),
    "ytf_plan_retune": (ctypes.c_int, [_vp, ctypes.POINTER(Tune)]),
    "ytf_plan_run": (ctypes.c_int, [_vp]),
    "ytf_plan_wait": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float)]),
    "ytf_plan_cache": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    "ytf_plan_info": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_long),
                                     ctypes.POINTER(ctypes.c_long)]),
    "ytf_plan_destroy": (ctypes.c_int, [_vp]),
    "ytf_gauss_legendre": (ctypes.c_int, [ctypes.c_int, _d, _d]),
    "ytf_gl_rule": (ctypes.c_int, [_vp, ctypes.c_int, _d, _d, ctypes.c_int, ctypes.c_int, _d, _d, _d]),
}

_lib = None


def lib():
    """Load libytf.so once; raise if it is absent (no silent fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libytf.so not found at {LIB_PATH}: build it with `python -m yellowthinfilms_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def ptr(a, t=_d):
    return None if a is None else a.ctypes.data_as(t)


def addr(a):
    """The address of a numpy array's data (for c_void_p descriptor fields); None for None."""
    return None if a is None else a.ctypes.data
