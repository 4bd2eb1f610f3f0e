"""ctypes binding of the C ABI in ``include/dmhm_b200.h``.

Loads the in-tree ``libdmhm_b200.so``; there is no fallback: if the library
is missing or was built without the CUDA kernels, importing the engine fails.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdmhm_b200.so")

HM_OK = 0
STATUS_NAMES = {
    1: "HM_ERR_ARGUMENT", 2: "HM_ERR_OOM", 3: "HM_ERR_CUDA", 4: "HM_ERR_UNSUPPORTED",
    5: "HM_ERR_NUMERICAL", 6: "HM_ERR_TIMEOUT", 7: "HM_ERR_INTERNAL",
}


class HMError(RuntimeError):
    """A non-zero status from the engine (the reference throws std::logic_error
    or std::runtime_error in the same places)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None

_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_U64 = C.c_uint64
_PI = C.POINTER(C.c_int)
_PD = C.POINTER(C.c_double)
_PI64 = C.POINTER(C.c_int64)
_PI32 = C.POINTER(C.c_int32)
_PU64 = C.POINTER(C.c_uint64)
_PF = C.POINTER(C.c_float)

# name -> argtypes (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "hm_last_error": [],
    "hm_version": [],
    "hm_context_create": [_I, _P, C.POINTER(_P)],
    "hm_context_destroy": [_P],
    "hm_context_synchronize": [_P],
    "hm_set_oversample": [_P, _I],
    "hm_get_oversample": [_P, _PI],
    "hm_set_compression_tolerance": [_P, _D],
    "hm_get_compression_tolerance": [_P, _PD],
    "hm_set_lcg_states": [_P, _U64, _U64],
    "hm_get_lcg_states": [_P, _PU64, _PU64],
    "hm_natural_to_hierarchical_map": [_I, _PI, _I, _PI],
    "hm_create_from_csr": [_P, _I, _PI, _I, _I, _I, _PI64, _PI32, _PD, C.POINTER(_P)],
    "hm_create_from_csr_complex": [_P, _I, _PI, _I, _I, _I, _PI64, _PI32, _PD, C.POINTER(_P)],
    "hm_is_complex": [_P, _PI],
    "hm_scale_complex": [_P, _D, _D],
    "hm_update_with": [_P, _D, _P],
    "hm_set_to_identity": [_P],
    "hm_conjugate_in_place": [_P],
    "hm_add_constant_to_diagonal_complex": [_P, _D, _D],
    "hm_conjugate": [_P, C.POINTER(_P)],
    "hm_transpose_complex": [_P, C.POINTER(_P)],
    "hm_packed_size": [_P, C.POINTER(C.c_size_t)],
    "hm_low_rank_product": [_P, _I, _D, _P, _I, _PD, _I, _PD, _I, _I, _PI],
    "hm_pack": [_P, _P, C.c_size_t, C.POINTER(C.c_size_t)],
    "hm_unpack": [_P, _I, _P, C.c_size_t, C.POINTER(_P)],
    "hm_multiply_dense_complex": [_P, _I, _D, _D, _P, _I, _D, _D, _P, _I, _I],
    "hm_multiply_dense_complex_host": [_P, _I, _D, _D, _PD, _I, _D, _D, _PD, _I, _I],
    "hm_destroy": [_P],
    "hm_info": [_P, _PI, _PI, _PI, _PI, _PI64, _PI64],
    "hm_structure": [_P, _PI, _PI, _PI, _PI],
    "hm_set_to_random": [_P],
    "hm_multiply_dense": [_P, _I, _D, _P, _I, _D, _P, _I, _I],
    "hm_multiply_dense_host": [_P, _I, _D, _PD, _I, _D, _PD, _I, _I],
    "hm_multiply_hmat": [_P, _D, _P, C.POINTER(_P)],
    "hm_multiply_hmat_update": [_P, _D, _P, _D, _P],
    "hm_estimate_two_norm": [_P, _D, _D, _PD],
    "hm_direct_invert": [_P],
    "hm_schulz_invert": [_P, _I, _D, _D, _D, _PI, _PD, _I, _PI],
    "hm_schulz_invert_mixed": [_P, _I, _D, _D, _D, _D, _PI, _PI, _PD, _I, _PI],
    "hm_set_low_precision": [_P, _I],
    "hm_copy": [_P, C.POINTER(_P)],
    "hm_transpose": [_P, C.POINTER(_P)],
    "hm_scale": [_P, _D],
    "hm_add_constant_to_diagonal": [_P, _D],
    "hm_multiply_vector_noalloc": [_P, _I, _D, _P, _D, _P],
    "hm_multiply_dense_tf32": [_P, _D, _P, _I, _D, _P, _I, _I],
    "hm_set_tf32_kernel": [_P, _I],
    "hm_tf32_kernel_choice": [_P, _P, _I, _I, _PI],
    "hm_set_fp64_split": [_P, _I],
    "hm_fp64_split_choice": [_P, _P, _I, _I, _PI],
    "hm_rank_feature_count": [],
    "hm_rank_param_count": [],
    "hm_rank_model_create": [_P, _U64, C.POINTER(_P)],
    "hm_rank_model_destroy": [_P],
    "hm_rank_model_set_params": [_P, _PF, _I],
    "hm_rank_model_get_params": [_P, _PF, _I],
    "hm_rank_model_loss_grad": [_P, _PF, _PF, _I, _PF, _PF],
    "hm_rank_model_train": [_P, _PF, _PF, _I, _I, C.c_float, _PF],
    "hm_rank_model_predict": [_P, _PF, _I, _PF],
    "hm_use_rank_model": [_P, _P, _I, _I],
    "hm_rank_log_enable": [_P, _I],
    "hm_rank_log_read": [_P, _PF, _PF, _I, _PI, _I],
    "hm_rank_stats": [_P, _PI64, _PI64, _PI64, _PI64],
    "hm_kernel_launches": [],
    "hm_measure_fp64_peak": [_I, _I, _I, _PD, _PD],
    "hm_check_bounded_wait": [_I, C.c_longlong, _PI],
    "hm_profile_enable": [_P, _I],
    "hm_profile_read": [_P, _I, C.c_char_p, _I, _PD, _PI64],
}
_RESTYPES = {"hm_last_error": C.c_char_p, "hm_version": C.c_int,
             "hm_rank_feature_count": C.c_int, "hm_rank_param_count": C.c_int,
             "hm_kernel_launches": C.c_ulonglong}


def lib():
    """The loaded library (raises if it is absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} not found: build it with `python dmhm_b200/build.py` "
                "(the engine has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPES.get(name, C.c_int)
        _lib = L
    return _lib


def check(status: int):
    if status != HM_OK:
        msg = lib().hm_last_error().decode(errors="replace")
        raise HMError(status, msg)
