"""The C-ABI library: it loads, exports every symbol include/fhe_b200.h declares,
and reports errors through status codes without a GPU."""
import ctypes
import os
import re

import pytest

from conftest import ROOT, HAS_GPU
from fhe_b200 import _lib

HEADER = os.path.join(ROOT, "include", "fhe_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^[A-Za-z_][\w \t\*]*?\b(fhe_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.SIGNATURES), "python bindings and header disagree"


def test_library_is_built_for_sm100a():
    out = os.popen(f"strings -a {_lib.LIB_PATH} | grep -c sm_100a").read().strip()
    assert out and int(out) >= 1


def test_null_handles_are_rejected():
    lib = _lib.load()
    assert lib.fhe_engine_info_get(None, None) == -5
    assert b"null handle" in lib.fhe_last_error()
    assert lib.fhe_data_destroy(None) == 0
    assert lib.fhe_engine_destroy(None) == 0


def test_config_default_matches_reference_defaults():
    cfg = _lib.FheConfig()
    _lib.load().fhe_config_default(ctypes.byref(cfg))
    assert (cfg.log_coeff_count, cfg.log_slot_count, cfg.special_prime_count, cfg.max_level,
            cfg.scheme_preset) == (14, -1, 1, -1, 1)


def test_invalid_config_fails_before_touching_the_device():
    lib = _lib.load()
    cfg = _lib.FheConfig(2, -1, 1, -1, 1)
    h = ctypes.c_void_p()
    assert lib.fhe_engine_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    assert b"too small" in lib.fhe_last_error()
    assert not h.value


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_engine_create_without_device_reports_cuda_error():
    lib = _lib.load()
    cfg = _lib.FheConfig(14, -1, 1, -1, 1)
    h = ctypes.c_void_p()
    rc = lib.fhe_engine_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == -3
    assert lib.fhe_last_error()
    assert not h.value
