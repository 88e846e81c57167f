"""fhe_relinearize_noalloc: the relinearization for callers that cannot allocate
device memory while they run (graph capture, fixed memory budgets).  It must give
the same words as fhe_relinearize, call after call, while taking every temporary
from the library's fixed device array.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from inputs import uniform_limbs

pytestmark = pytest.mark.gpu

NTT, SPECIAL = 2, 16


def _noalloc(e, ct, mid, key, key_mid, out):
    from fhe_b200 import _lib

    lib = _lib.load()
    kinfo = key.info()
    rc = lib.fhe_relinearize_noalloc(
        e.handle, ctypes.cast(ct.device_pointer(), _lib._i64p), mid,
        ctypes.cast(key.device_pointer(), _lib._i64p), key_mid, kinfo["polys"],
        ctypes.cast(out.device_pointer(), _lib._i64p))
    return rc, lib.fhe_last_error().decode()


def test_noalloc_relinearize_matches_relinearize_twice():
    from fhe_b200 import Engine, RELINEARIZATION_KEY

    e = Engine(log_coeff_count=14, special_prime_count=1)  # the reference's default config
    mid = e.moduli_id(e.max_key_switching_level)
    L = e.chains(mid)
    rng = np.random.default_rng(2024)
    key = uniform_limbs(rng, e.moduli[mid:], 2 * e.partition_count(mid), e.coeff_count)
    rk = e.upload(key, mid, NTT | SPECIAL, RELINEARIZATION_KEY)
    out = e.upload(np.zeros((2, L, e.coeff_count), dtype=np.int64), mid)
    for call in range(2):
        ct = e.upload(uniform_limbs(rng, e.moduli[mid:mid + L], 3, e.coeff_count), mid, NTT)
        rc, msg = _noalloc(e, ct, mid, rk, mid, out)
        assert rc == 0, msg
        want = e.relinearize(ct, rk).download()
        assert np.array_equal(out.download(), want), f"call {call}"
    e.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from fhe_b200 import Engine, RELINEARIZATION_KEY

    e = Engine(log_coeff_count=16, special_prime_count=4)
    mid = e.moduli_id(e.max_key_switching_level)
    L = e.chains(mid)
    rng = np.random.default_rng(7)
    key = uniform_limbs(rng, e.moduli[mid:], 2 * e.partition_count(mid), e.coeff_count)
    rk = e.upload(key, mid, NTT | SPECIAL, RELINEARIZATION_KEY)
    ct = e.upload(uniform_limbs(rng, e.moduli[mid:mid + L], 3, e.coeff_count), mid, NTT)
    out = e.upload(np.zeros((2, L, e.coeff_count), dtype=np.int64), mid)
    rc, msg = _noalloc(e, ct, mid, rk, mid, out)
    assert rc == -1
    assert "scratch words" in msg
    e.close()
