import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine")


def _has_gpu() -> bool:
    try:
        import ctypes

        cudart = ctypes.CDLL("libcudart.so")
        count = ctypes.c_int(0)
        return cudart.cudaGetDeviceCount(ctypes.byref(count)) == 0 and count.value > 0
    except OSError:
        try:
            import torch

            return torch.cuda.is_available()
        except Exception:
            return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ref_ops():
    return load_golden("ref_ops.json")


@pytest.fixture(scope="module")
def engines():
    """Engines on cuda:0, one per (log_n, special prime count, preset), per module."""
    from fhe_b200 import Engine

    cache = {}

    def get(log_n, K, preset, log_slot=-1):
        key = (log_n, K, preset, log_slot)
        if key not in cache:
            cache[key] = Engine(log_coeff_count=log_n, special_prime_count=K, scheme_preset=preset,
                                log_slot_count=log_slot)
        return cache[key]

    yield get
    for e in cache.values():
        e.close()
