"""fhe_relinearize_noalloc: the relinearization for callers that cannot allocate
device memory while they run (an application allocator that owns the GPU's memory,
real-time loops that cannot take an allocation's implicit synchronisation, stream
callbacks).  It must give the same words as fhe_relinearize, call after call, while
taking every temporary from the library's fixed device array and allocating no
device memory.  This file is collected last on purpose: if it fails, a run that
stops at the first failure has already run every other test."""
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


def _free_device_bytes():
    """Free memory of the current device as the CUDA runtime reports it (the
    engine library has loaded libcudart.so.12 already, so this is the same one)."""
    cudart = ctypes.CDLL("libcudart.so.12")
    free, total = ctypes.c_size_t(0), ctypes.c_size_t(0)
    assert cudart.cudaDeviceSynchronize() == 0
    assert cudart.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


# (log_n, special primes, tensor-core mode of the engine's own relinearize, text
# moduli ids); the key is made at the key-switching level.  K = 1 has one-limb
# partitions (the reference's default engine); K = 3 has partitions of 2 and 3
# limbs, so the Garner constants are non-trivial, and texts below the key's level
# read the key through a partition offset; K = 4 compares against fhe_relinearize
# with both base conversions on the INT8 tensor pipe.
CASES = [(14, 1, 2, [1, 4]), (14, 3, 2, [1, 2, 3]), (14, 4, 1, [1, 2])]


@pytest.mark.parametrize("log_n,K,mode,mids", CASES, ids=lambda v: str(v))
def test_noalloc_relinearize_matches_relinearize_twice(log_n, K, mode, mids):
    from fhe_b200 import Engine, RELINEARIZATION_KEY

    e = Engine(log_coeff_count=log_n, special_prime_count=K)
    e.set_tensor_cores(mode)
    key_mid = e.moduli_id(e.max_key_switching_level)
    rng = np.random.default_rng(2024 + K)
    key = uniform_limbs(rng, e.moduli[key_mid:], 2 * e.partition_count(key_mid), e.coeff_count)
    rk = e.upload(key, key_mid, NTT | SPECIAL, RELINEARIZATION_KEY)
    for mid in mids:
        L = e.chains(mid)
        out = e.upload(np.zeros((2, L, e.coeff_count), dtype=np.int64), mid)
        for call in range(2):
            ct = e.upload(uniform_limbs(rng, e.moduli[mid:mid + L], 3, e.coeff_count), mid, NTT)
            rc, msg = _noalloc(e, ct, mid, rk, key_mid, out)
            assert rc == 0, msg
            want = e.relinearize(ct, rk).download()
            assert np.array_equal(out.download(), want), f"moduli id {mid}, call {call}"
    e.close()


def test_noalloc_relinearize_allocates_no_device_memory():
    from fhe_b200 import Engine, RELINEARIZATION_KEY

    e = Engine(log_coeff_count=14, special_prime_count=3)
    mid = e.moduli_id(e.max_key_switching_level)
    L = e.chains(mid)
    rng = np.random.default_rng(99)
    key = uniform_limbs(rng, e.moduli[mid:], 2 * e.partition_count(mid), e.coeff_count)
    rk = e.upload(key, mid, NTT | SPECIAL, RELINEARIZATION_KEY)
    ct = e.upload(uniform_limbs(rng, e.moduli[mid:mid + L], 3, e.coeff_count), mid, NTT)
    out = e.upload(np.zeros((2, L, e.coeff_count), dtype=np.int64), mid)
    rc, msg = _noalloc(e, ct, mid, rk, mid, out)  # the first call resolves the array
    assert rc == 0, msg
    for _ in range(3):
        before = _free_device_bytes()
        rc, msg = _noalloc(e, ct, mid, rk, mid, out)
        assert rc == 0, msg
        assert _free_device_bytes() == before
    assert np.array_equal(out.download(), e.relinearize(ct, rk).download())
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
