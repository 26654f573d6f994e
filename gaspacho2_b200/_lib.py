"""ctypes binding of libgpl_b200.so (include/gpl.h). There is no fallback: if the library is
missing or does not load, every call raises."""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libgpl_b200.so")

GPL_OK = 0
ERRORS = {-1: "GPL_ERR_ARG", -2: "GPL_ERR_CUDA", -3: "GPL_ERR_ALLOC", -4: "GPL_ERR_STATE", -5: "GPL_ERR_NAN",
          -6: "GPL_ERR_FORMAT", -7: "GPL_ERR_IO",
          -8: "GPL_ERR_LIMIT", -9: "GPL_ERR_TIMEOUT"}
PREC = {"fp64": 0, "bf16x3": 1}
DE_NULL, DE_FULL = -2, -1  # gpl_de_model's model codes besides a latent dimension

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_vp = ctypes.c_void_p

# name -> (restype, argtypes); every entry point returns int except gpl_last_error and
# gpl_ta_equispaced
SIGNATURES = {
    "gpl_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, _vp]),
    "gpl_destroy": (ctypes.c_int, [_vp]),
    "gpl_last_error": (ctypes.c_char_p, [_vp]),
    "gpl_set_precision": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gpl_set_option": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_int64]),
    "gpl_get_option": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]),
    "gpl_tuning": (ctypes.c_int, [_vp, ctypes.c_char_p, _ip, _ip, _dp, ctypes.c_int, _ip]),
    "gpl_load_counts": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int64, _ip, _ip, _dp]),
    "gpl_load_design": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _ip, _ip, _vp, ctypes.c_int64, ctypes.c_int,
                                       ctypes.c_int]),
    "gpl_set_size_factors": (ctypes.c_int, [_vp, _dp]),
    "gpl_dims": (ctypes.c_int, [_vp, _ip]),
    "gpl_init_params": (ctypes.c_int, [_vp]),
    "gpl_set_params": (ctypes.c_int, [_vp] + [_dp] * 6),
    "gpl_get_params": (ctypes.c_int, [_vp] + [_dp] * 6),
    "gpl_set_beta": (ctypes.c_int, [_vp, _dp]),
    "gpl_get_beta": (ctypes.c_int, [_vp, _dp]),
    "gpl_kernel_mats": (ctypes.c_int, [_vp]),
    "gpl_glm_init": (ctypes.c_int, [_vp]),
    "gpl_expand_delta": (ctypes.c_int, [_vp]),
    "gpl_gram": (ctypes.c_int, [_vp]),
    "gpl_irls_sweep": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "gpl_irls": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "gpl_objective_after_irls": (ctypes.c_int, [_vp, _dp]),
    "gpl_objective": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "gpl_gradient": (ctypes.c_int, [_vp, _dp]),
    "gpl_lbfgs_update": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "gpl_downdate": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]),
    "gpl_beta_from_tilde": (ctypes.c_int, [_vp]),
    "gpl_fit": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _ip, _dp, ctypes.c_int]),
    "gpl_fit_outer": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _ip, _dp, ctypes.c_int]),
    "gpl_score_stats": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp]),
    "gpl_de_model": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gpl_vc_fit": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int, _ip]),
    "gpl_de_irls": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, _dp, _ip, _dp, ctypes.c_int]),
    "gpl_ta_equispaced": (None, [ctypes.c_int, ctypes.c_int, _dp]),
    "gpl_evaluate": (ctypes.c_int, [_vp, _dp, ctypes.c_int64, _dp, _dp]),
    "gpl_evaluate_device": (ctypes.c_int, [_vp]),
    "gpl_get": (ctypes.c_int, [_vp, ctypes.c_char_p, _dp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "gpl_profile_enable": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gpl_profile_reset": (ctypes.c_int, [_vp]),
    "gpl_profile_read": (ctypes.c_int, [_vp, ctypes.c_char_p, _dp, ctypes.POINTER(ctypes.c_int64)]),
    "gpl_launch_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "gpl_sync": (ctypes.c_int, [_vp]),
    "gpl_wait_probe": (ctypes.c_int, [_vp, ctypes.c_int64]),
    "gpl_init_latent": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, _dp, _dp]),
    "gpl_cis_stats": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _dp, _dp]),
    "gpl_place_cells": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp, _ip]),
    "gpl_cell_objective": (ctypes.c_int, [_vp, _dp, _dp, _dp]),
    "gpl_enc_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_uint64]),
    "gpl_enc_destroy": (ctypes.c_int, [_vp]),
    "gpl_enc_last_error": (ctypes.c_char_p, [_vp]),
    "gpl_enc_set_cells": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64, _ip, _ip, _dp,
                                         _dp, _ip, _ip]),
    "gpl_enc_set_targets": (ctypes.c_int, [_vp, _dp]),
    "gpl_enc_n_params": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "gpl_enc_get_params": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float)]),
    "gpl_enc_set_params": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float)]),
    "gpl_enc_grads": (ctypes.c_int, [_vp, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_float)]),
    "gpl_enc_train": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_uint64, _dp]),
    "gpl_enc_predict": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp]),
    "gpl_enc_launch_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "gpl_kernel_mats_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp,
                                               _vp, _vp]),
}

_lib = None


class GplError(RuntimeError):
    pass


def load():
    """Loads the in-tree library; raises if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GplError(f"{LIB_PATH} is not built: run `python -m gaspacho2_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int, ctx=None, what: str = "") -> None:
    if rc != GPL_OK:
        msg = ""
        if ctx is not None:
            m = load().gpl_last_error(ctx)
            msg = m.decode() if m else ""
        raise GplError(f"{what}: {ERRORS.get(rc, rc)} {msg}".strip())
