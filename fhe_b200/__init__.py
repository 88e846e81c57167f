"""fhe_b200: a B200-native CKKS engine with the DESILO FHE engine API.

The compute path is hand-written sm_100a CUDA behind the C ABI declared in
include/fhe_b200.h; :mod:`fhe_b200.engine` mirrors the reference engine's API in
Python over that ABI.
"""
from .engine import (  # noqa: F401
    CKKS_40_60_DEFAULT,
    CKKS_40_60_DEFAULT_ENGINE_TEST,
    CKKS_54_60_BOOTSTRAP,
    CKKS_54_60_BOOTSTRAP_ENGINE_TEST,
    COMPLEX,
    CONJUGATION_KEY,
    FIXED_ROTATION_KEY,
    INCLUDE_SPECIAL,
    KEY_SWITCHING_KEY,
    NONE,
    NTT_FORM,
    RELINEARIZATION_KEY,
    RESCALED,
    UNIT_CIPHERTEXT,
    UNIT_PLAINTEXT,
    Data,
    Engine,
    FheError,
)
