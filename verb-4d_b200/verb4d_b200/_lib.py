"""ctypes binding of libverb4d_b200.so (the C ABI declared in include/verb4d_b200.h).

The shared library is built in-tree (``make -C verb-4d_b200/csrc``).  There is
no CPU fallback: if the library or a CUDA device is missing, calls fail with
an exception.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libverb4d_b200.so")

VERB_OK = 0
VERB_PREC_FP64 = 0
VERB_PREC_MIXED = 1
STATUS_NAMES = {
    0: "VERB_OK", 1: "VERB_ERR_PIVOT", 2: "VERB_ERR_ARG", 3: "VERB_ERR_CFL", 4: "VERB_ERR_BC",
    5: "VERB_ERR_TENSOR", 6: "VERB_ERR_NAN", 7: "VERB_ERR_CUDA", 8: "VERB_ERR_NOMEM",
    9: "VERB_ERR_GRID", 10: "VERB_TIMEOUT", 11: "VERB_ERR_SIZE", 12: "VERB_ERR_IO",
}
VERB_GUESS_ZERO, VERB_GUESS_PREV, VERB_GUESS_CNN = 0, 1, 2
CONV_ARITH = {"exact": 0, "fma": 1, "stream": 2}
GUESS_IDS = {"zero": VERB_GUESS_ZERO, "prev": VERB_GUESS_PREV, "cnn": VERB_GUESS_CNN}


class KrylovStats(C.Structure):
    _fields_ = [("systems", C.c_longlong), ("fallbacks", C.c_longlong),
                ("inner_iterations", C.c_longlong), ("solved_iterations", C.c_longlong),
                ("outer_passes", C.c_longlong),
                ("max_rel_residual", C.c_double), ("guess_rel_residual", C.c_double)]

# 4-D fields (verb_field)
F_PSD, F_P, F_R, F_V, F_K, F_L, F_DLL, F_DVV, F_DKK, F_DVK, F_VP, F_VR, F_G_LOCAL, F_G_RADIAL, \
    F_G_CONV, F_SOURCES, F_LOSS_LOCAL, F_LOSS_RADIAL, F_LOSS_CONV = range(19)
FIELD_IDS = {
    "psd": F_PSD, "Pg": F_P, "Rg": F_R, "Vg": F_V, "Kg": F_K, "Lg": F_L, "DLL": F_DLL, "DVV": F_DVV,
    "DKK": F_DKK, "DVK": F_DVK, "VP": F_VP, "VR": F_VR, "G_local": F_G_LOCAL,
    "G_radial": F_G_RADIAL, "G_conv": F_G_CONV, "S": F_SOURCES, "loss_local": F_LOSS_LOCAL,
    "loss_radial": F_LOSS_RADIAL, "loss_conv": F_LOSS_CONV,
}
# 3-D boundary arrays (verb_bc_field)
BC_FIELDS = ("Pl", "Pu", "Rl", "Ru", "Ll", "Lu", "Vl", "Vu", "Kl", "Ku")


class VerbError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)} ({status})")


class Timing(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("convection_ms", "radial_ms", "radial_factor_ms",
                                            "local_ms", "local_factor_ms", "local_solve_ms",
                                            "reduce_ms", "kf_ms")] + \
               [(n, C.c_longlong) for n in ("steps", "local_solve_launches",
                                              "local_factor_launches", "kernel_launches")]


_dp = C.POINTER(C.c_double)
_lp = C.POINTER(C.c_long)
_ip = C.POINTER(C.c_int)
_i32p = C.POINTER(C.c_int32)
_llp = C.POINTER(C.c_longlong)
_vp = C.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "verb_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
    "verb_destroy": (C.c_int, [_vp]),
    "verb_device_bytes": (C.c_int, [_vp, C.POINTER(C.c_size_t)]),
    "verb_upload_field": (C.c_int, [_vp, C.c_int, _dp]),
    "verb_upload_field_device": (C.c_int, [_vp, C.c_int, _vp]),
    "verb_set_field_scale": (C.c_int, [_vp, C.c_int, C.c_double]),
    "verb_upload_bc": (C.c_int, [_vp, C.c_int, _dp]),
    "verb_set_bc_types": (C.c_int, [_vp, _ip]),
    "verb_set_options": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int]),
    "verb_invalidate_lu": (C.c_int, [_vp]),
    "verb_remap_L": (C.c_int, [_vp, _dp]),
    "verb_cnn_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.POINTER(C.c_int), C.c_int, C.c_int,
                                  C.c_int, _vp]),
    "verb_cnn_destroy": (C.c_int, [_vp]),
    "verb_cnn_param_count": (C.c_int, [_vp, C.POINTER(C.c_longlong)]),
    "verb_cnn_set_params": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "verb_cnn_get_params": (C.c_int, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "verb_cnn_forward": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "verb_cnn_train_step": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_float, C.POINTER(C.c_float)]),
    "verb_local_krylov": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, _vp, C.c_int,
                                    C.c_double, C.c_int, C.c_int, C.c_double, C.c_double, _vp]),
    "verb_local_triples": (C.c_int, [_vp, C.c_double, C.c_double, _vp, _vp]),
    "verb_cnn_backward_step": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_float]),
    "verb_set_krylov_preconditioner": (C.c_int, [_vp, _vp]),
    "verb_local_precond_inputs": (C.c_int, [_vp, C.c_double, C.c_double, _vp, _vp]),
    "verb_precond_loss_grad": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp,
                                         C.POINTER(C.c_float), _vp]),
    "verb_set_convection_arith": (C.c_int, [_vp, C.c_int]),
    "verb_set_step_graph": (C.c_int, [_vp, C.c_int]),
    "verb_local_solve_variants": (C.c_int, [C.POINTER(C.c_int)]),
    "verb_local_solve_variant": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                           C.POINTER(C.c_int)]),
    "verb_local_solve_variant_window": (C.c_int, [C.c_int, C.POINTER(C.c_int)]),
    "verb_set_local_solve_variant": (C.c_int, [_vp, C.c_int]),
    "verb_autotune_local_solve": (C.c_int, [_vp, C.c_double, C.c_double, _dp,
                                            C.POINTER(C.c_int)]),
    "verb_assimilate_convection": (C.c_int, [_vp, _dp, C.c_double, C.c_double, C.c_double, C.c_int,
                                             C.c_double, C.c_int, C.c_int, C.c_int]),
    "verb_convection_da_state": (C.c_int, [_vp, C.c_int, C.c_int, _dp, _dp]),
    "verb_set_local_trim": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "verb_estimate_device_bytes": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.c_longlong, C.POINTER(C.c_size_t)]),
    "verb_write_field_pltb": (C.c_int, [_vp, C.c_int, C.c_char_p, C.c_int]),
    "verb_output_wait": (C.c_int, [_vp]),
    "verb_read_field_pltb": (C.c_int, [_vp, C.c_int, C.c_char_p]),
    "verb_append_lst": (C.c_int, [C.c_char_p, C.c_double, C.c_char_p]),
    "verb_field_add_component": (C.c_int, [_vp, C.c_int, _dp, C.POINTER(C.c_int)]),
    "verb_field_set_merge": (C.c_int, [_vp, C.c_int, C.c_int]),
    "verb_component_queue_data": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, _dp]),
    "verb_component_queue_scale": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_double]),
    "verb_component_queue_limit": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                             C.c_double]),
    "verb_update_fields": (C.c_int, [_vp, C.c_double, C.POINTER(C.c_uint)]),
    "verb_set_local_precision": (C.c_int, [_vp, C.c_int, C.c_int]),
    "verb_local_refinement": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "verb_download_psd": (C.c_int, [_vp, _dp]),
    "verb_download_field": (C.c_int, [_vp, C.c_int, _dp]),
    "verb_field_device_ptr": (C.c_int, [_vp, C.c_int, C.POINTER(_dp)]),
    "verb_convection": (C.c_int, [_vp, C.c_double]),
    "verb_radial": (C.c_int, [_vp, C.c_double]),
    "verb_local": (C.c_int, [_vp, C.c_double, C.c_double]),
    "verb_clamp_positive": (C.c_int, [_vp]),
    "verb_step": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _llp]),
    "verb_negative_count": (C.c_int, [_vp, _llp]),
    "verb_tensor_check": (C.c_int, [_vp, _dp]),
    "verb_field_maxabs": (C.c_int, [_vp, C.c_int, _ip, _dp]),
    "verb_sync": (C.c_int, [_vp]),
    "verb_set_timing": (C.c_int, [_vp, C.c_int]),
    "verb_get_timing": (C.c_int, [_vp, C.POINTER(Timing)]),
    "verb_convection_substeps": (C.c_int, [_vp, _ip]),
    "verb_local_pivots": (C.c_int, [_vp, _i32p]),
    "verb_local_factor_lapack": (C.c_int, [_vp, C.c_int, C.c_int, _dp, _lp]),
    "verb_assimilate_radial": (C.c_int, [_vp, _dp, C.c_double, C.c_double, C.c_double, C.c_int]),
    "verb_tridag": (C.c_int, [_dp, _dp, _dp, _dp, _dp, C.c_long]),
    "verb_diffusion_1d": (C.c_int, [_dp, _dp, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                    _dp, _dp, _dp, _dp, C.c_double]),
    "verb_diffusion_2d": (C.c_int, [_dp, _dp, _dp, C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_int,
                                    C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                    C.c_double, C.c_double, _dp, _lp, C.c_int]),
    "verb_convection_1d": (C.c_int, [_dp, _dp, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                     _dp, C.c_double]),
    "verb_convection_2d": (C.c_int, [_dp, _dp, _dp, C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_int,
                                     C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp,
                                     C.c_double]),
    "verb_convection_2d_noalloc": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp,
                                             C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp,
                                             _vp, _vp, C.c_double, _vp]),
    "verb_version": (C.c_char_p, []),
    "verb_status_string": (C.c_char_p, [C.c_int]),
}

_lib = None


def load(path: str | None = None):
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(
            f"{p} is missing: build it with `make -C verb-4d_b200/csrc` (there is no CPU fallback)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status: int, what: str) -> None:
    if status != VERB_OK:
        raise VerbError(status, what)
