"""Loader and ctypes signatures of the engine's C ABI (include/fhe_b200.h).

The shared library is built in-tree by ``python -m fhe_b200.build``.  There is no
fallback: if it is missing, importing the engine raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfhe_b200.so")

FHE_OK = 0
STATUS_NAMES = {
    -1: "FHE_ERR_INVALID_ARGUMENT",
    -2: "FHE_ERR_RUNTIME",
    -3: "FHE_ERR_CUDA",
    -4: "FHE_ERR_OUT_OF_MEMORY",
    -5: "FHE_ERR_NULL_HANDLE",
    -6: "FHE_ERR_UNSUPPORTED",
}

# Every symbol include/fhe_b200.h declares, with (restype, argtypes).
_vp = ctypes.c_void_p
_i = ctypes.c_int
_pp = ctypes.POINTER(ctypes.c_void_p)
_ip = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)


class FheConfig(ctypes.Structure):
    _fields_ = [("log_coeff_count", ctypes.c_int), ("log_slot_count", ctypes.c_int),
                ("special_prime_count", ctypes.c_int), ("max_level", ctypes.c_int),
                ("scheme_preset", ctypes.c_int)]


class FheEngineInfo(ctypes.Structure):
    _fields_ = [("coeff_count", ctypes.c_int), ("slot_count", ctypes.c_int),
                ("chain_count", ctypes.c_int), ("prime_count", ctypes.c_int),
                ("special_prime_count", ctypes.c_int), ("full_level", ctypes.c_int),
                ("max_level", ctypes.c_int), ("max_key_switching_level", ctypes.c_int),
                ("scale_bit_length", ctypes.c_int)]


class FheDataInfo(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("flag", ctypes.c_int), ("moduli_id", ctypes.c_int),
                ("level", ctypes.c_int), ("polys", ctypes.c_int), ("chains", ctypes.c_int),
                ("delta", ctypes.c_int), ("ckks_scale", ctypes.c_longdouble)]


SIGNATURES = {
    "fhe_last_error": (ctypes.c_char_p, []),
    "fhe_config_default": (None, [ctypes.POINTER(FheConfig)]),
    "fhe_engine_set_profiling": (_i, [_vp, _i]),
    "fhe_engine_profile_report": (_i, [_vp, ctypes.c_char_p, _i]),
    "fhe_engine_profile_reset": (_i, [_vp]),
    "fhe_kernel_launch_count": (ctypes.c_ulonglong, []),
    "fhe_parameters_query":(_i, [ctypes.POINTER(FheConfig), ctypes.POINTER(FheEngineInfo),
                                  ctypes.POINTER(ctypes.c_uint64), _i]),
    "fhe_parameters_tables": (_i, [ctypes.POINTER(FheConfig), ctypes.POINTER(ctypes.c_uint64),
                                   _i64p, _i64p, _i64p, _i64p]),
    "fhe_engine_create": (_i, [ctypes.POINTER(FheConfig), _pp]),
    "fhe_engine_destroy": (_i, [_vp]),
    "fhe_engine_info_get": (_i, [_vp, ctypes.POINTER(FheEngineInfo)]),
    "fhe_engine_moduli": (_i, [_vp, ctypes.POINTER(ctypes.c_uint64), _i]),
    "fhe_engine_moduli_id": (_i, [_vp, _i, ctypes.POINTER(ctypes.c_int)]),
    "fhe_engine_synchronize": (_i, [_vp]),
    "fhe_engine_set_stream": (_i, [_vp, _vp]),
    "fhe_data_upload": (_i, [_vp, _i, _i, _i, _i, ctypes.c_longdouble, _i64p, _pp]),
    "fhe_data_download": (_i, [_vp, _i64p]),
    "fhe_data_download_async": (_i, [_vp, _i64p]),
    "fhe_data_info_get": (_i, [_vp, ctypes.POINTER(FheDataInfo)]),
    "fhe_data_set_delta": (_i, [_vp, _i]),
    "fhe_data_device_pointer": (_i, [_vp, ctypes.POINTER(_i64p)]),
    "fhe_data_destroy": (_i, [_vp]),
    "fhe_multiply": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_multiply_relinearize": (_i, [_vp, _vp, _vp, _vp, _pp]),
    "fhe_relinearize": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_rescale": (_i, [_vp, _vp, _pp]),
    "fhe_multiply_relinearize_rescale": (_i, [_vp, _vp, _vp, _vp, _pp]),
    "fhe_to_ntt": (_i, [_vp, _vp, _pp]),
    "fhe_to_intt": (_i, [_vp, _vp, _pp]),
    "fhe_level_down": (_i, [_vp, _vp, _i, _pp]),
    "fhe_rotate": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_rotate_with_keys": (_i, [_vp, _vp, ctypes.POINTER(_vp), _i, _i, _i, _pp]),
    "fhe_rotate_plaintext": (_i, [_vp, _vp, _i, _pp]),
    "fhe_conjugate": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_conjugate_plaintext": (_i, [_vp, _vp, _pp]),
    "fhe_switch_key": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_encode": (_i, [_vp, _f64p, _f64p, _i, _i, _i, _pp]),
    "fhe_create_small_bootstrap_key": (_i, [_vp, _vp, _pp, _pp]),
    "fhe_bootstrap": (_i, [_vp, _vp, _vp, _vp, ctypes.POINTER(_vp), _i, _vp, _vp, _i, _pp]),
    "fhe_rotate_batch": (_i, [_vp, _vp, ctypes.POINTER(_vp), _i, _pp]),
    "fhe_data_serialized_size": (_i, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "fhe_data_serialize": (_i, [_vp, _vp, ctypes.c_uint64]),
    "fhe_data_deserialize": (_i, [_vp, _vp, ctypes.c_uint64, _pp]),
    "fhe_ntt_tuning_set": (_i, [_i, _i, _i, _i]),
    "fhe_ntt_tuning_get": (_i, [_i, _ip, _ip, _ip]),
    "fhe_engine_set_tensor_cores": (_i, [_vp, _i]),
    "fhe_engine_set_tensor_core_wait_limit": (_i, [_vp, ctypes.c_longlong]),
    "fhe_engine_set_graphs": (_i, [_vp, _i]),
    "fhe_engine_set_fused_bsgs": (_i, [_vp, _i]),
    "fhe_engine_set_value_transforms": (_i, [_vp, _i]),
    "fhe_engine_set_concurrency": (_i, [_vp, _i]),
    "fhe_multiply_relinearize_rescale_batch": (_i, [_vp, _i, ctypes.POINTER(_vp),
                                                   ctypes.POINTER(_vp), _vp, ctypes.POINTER(_vp)]),
    "fhe_bootstrap_batch": (_i, [_vp, _i, ctypes.POINTER(_vp), _vp, _vp, _vp,
                                ctypes.POINTER(_vp)]),
    "fhe_engine_graph_counts": (_i, [_vp, _ip, _ip]),
    "fhe_multiply_rotate_batch": (_i, [_vp, _i, ctypes.POINTER(_vp), ctypes.POINTER(_vp), _vp,
                                       ctypes.POINTER(_vp), _pp]),
    "fhe_create_bootstrap_key": (_i, [_vp, _vp, _i, ctypes.c_char_p, _pp]),
    "fhe_bootstrap_key_destroy": (_i, [_vp]),
    "fhe_bootstrap_key_info": (_i, [_vp, _ip, _ip, _ip, ctypes.POINTER(ctypes.c_uint64)]),
    "fhe_bootstrap_key_deltas": (_i, [_vp, _ip, _i, _ip]),
    "fhe_bootstrap_key_rotation_key": (_i, [_vp, _vp, _i, _pp]),
    "fhe_bootstrap_key_stage": (_i, [_vp, _i, _i, _ip, _ip, _ip]),
    "fhe_bootstrap_key_diagonal": (_i, [_vp, _vp, _i, _i, _i, _i, _pp]),
    "fhe_bootstrap_key_small": (_i, [_vp, _vp, _pp, _pp]),
    "fhe_bootstrap_with_key": (_i, [_vp, _vp, _vp, _vp, _vp, _pp]),
    "fhe_rotate_with_bootstrap_key": (_i, [_vp, _vp, _vp, _i, _pp]),
    "fhe_add": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_subtract": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_add_plaintext": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_subtract_plaintext": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_subtract_from_plaintext": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_multiply_plaintext": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_add_scalar": (_i, [_vp, _vp, ctypes.c_double, _pp]),
    "fhe_subtract_scalar": (_i, [_vp, _vp, ctypes.c_double, _pp]),
    "fhe_multiply_scalar": (_i, [_vp, _vp, ctypes.c_double, _pp]),
    "fhe_multiply_integer": (_i, [_vp, _vp, ctypes.c_longlong, _pp]),
    "fhe_negate": (_i, [_vp, _vp, _pp]),
    "fhe_square": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_engine_seed": (_i, [_vp, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint8)]),
    "fhe_create_secret_key": (_i, [_vp, _i, _pp]),
    "fhe_create_secret_key_from": (_i, [_vp, _i64p, _i, _i, _pp]),
    "fhe_create_sparse_secret_key": (_i, [_vp, _i, _i, _pp]),
    "fhe_create_public_key": (_i, [_vp, _vp, _i, _pp]),
    "fhe_create_relinearization_key": (_i, [_vp, _vp, _i, _pp]),
    "fhe_create_fixed_rotation_key": (_i, [_vp, _vp, _i, _i, _i, _pp]),
    "fhe_create_rotation_keys": (_i, [_vp, _vp, _i, ctypes.POINTER(_vp), _i,
                                      ctypes.POINTER(ctypes.c_int)]),
    "fhe_create_conjugation_key": (_i, [_vp, _vp, _i, _pp]),
    "fhe_encrypt": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_decrypt": (_i, [_vp, _vp, _vp, _pp]),
    "fhe_decode": (_i, [_vp, _vp, _f64p, _f64p]),
    "fhe_mont_mult_limbs": (_i, [_vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _i, _i, _i,
                                 ctypes.c_longlong]),
    "fhe_ntt_limbs": (_i, [_vp, _i64p, _i, _i, _i, ctypes.c_longlong, _i]),
    "fhe_relinearize_noalloc": (_i, [_vp, _i64p, _i, _i64p, _i, _i, _i64p]),
}

_lib = None


def load():
    """Load libfhe_b200.so and bind every C-ABI symbol (raises if missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing; build it with `python -m fhe_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
        install_ntt_tuning(lib)
    return _lib


TUNING_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ntt_tuning.json")


def install_ntt_tuning(lib, path: str = TUNING_PATH) -> int:
    """Installs the NTT shapes measured by fhe_b200.autotune (if the file exists);
    returns how many transform sizes were set."""
    if not os.path.exists(path):
        return 0
    import json

    with open(path) as f:
        table = json.load(f)
    count = 0
    for log_n, t in table.get("ntt", {}).items():
        if lib.fhe_ntt_tuning_set(int(log_n), t["s_second"], t["first_columns_log"],
                                  t["second_tile_log"]) == 0:
            count += 1
    return count


class FheError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


def check(status: int) -> None:
    if status != FHE_OK:
        msg = load().fhe_last_error().decode()
        if status == -1:
            raise FheInvalidArgument(status, msg)
        raise FheError(status, msg)


class FheInvalidArgument(FheError, ValueError):
    pass
