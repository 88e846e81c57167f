"""NTT shape tuning: the ABI rejects shapes the kernels cannot run, the package
installs the measured table, and (on the GPU) every shape gives the same words."""
import ctypes

import numpy as np
import pytest

from fhe_b200 import _lib
from inputs import uniform_limbs


def get(lib, log_n):
    v = [ctypes.c_int() for _ in range(3)]
    assert lib.fhe_ntt_tuning_get(log_n, *[ctypes.byref(x) for x in v]) == 0
    return tuple(x.value for x in v)


def test_invalid_shapes_are_rejected_and_leave_the_table_alone():
    lib = _lib.load()
    before = get(lib, 16)
    assert lib.fhe_ntt_tuning_set(16, 3, 2, 12) != 0   # outer pass of 13 stages
    assert lib.fhe_ntt_tuning_set(16, 8, 9, 12) != 0   # more columns than the stride
    assert lib.fhe_ntt_tuning_set(16, 8, 4, 15) != 0   # tile beyond shared memory
    assert lib.fhe_ntt_tuning_set(11, 5, 2, 11) != 0   # single-pass size
    assert get(lib, 16) == before


def test_the_measured_table_is_installed():
    lib = _lib.load()
    import json

    table = json.load(open(_lib.TUNING_PATH))["ntt"]
    assert _lib.install_ntt_tuning(lib) == len(table)
    for log_n, t in table.items():
        assert get(lib, int(log_n)) == (t["s_second"], t["first_columns_log"], t["second_tile_log"])


@pytest.mark.gpu
@pytest.mark.parametrize("log_n,K,shapes", [
    (14, 1, [(6, 2, 11), (7, 4, 12), (9, 5, 13)]),
    (16, 10, [(5, 3, 11), (8, 4, 12), (11, 5, 11)]),
])
def test_every_shape_gives_the_same_words(engines, log_n, K, shapes):
    lib = _lib.load()
    e = engines(log_n, K, 1)
    mid = e.moduli_id(e.max_key_switching_level)
    rng = np.random.default_rng(600 + log_n)
    q = e.moduli[mid:e.chain_count]
    a, b = uniform_limbs(rng, q, 2, e.coeff_count), uniform_limbs(rng, q, 2, e.coeff_count)
    key = uniform_limbs(rng, e.moduli[mid:], 2 * e.partition_count(mid), e.coeff_count)
    rk = e.upload(key, mid, 2 | 16, 3)
    saved = get(lib, log_n)
    outs = []
    try:
        for shape in shapes:
            assert lib.fhe_ntt_tuning_set(log_n, *shape) == 0
            outs.append(e.multiply_relinearize_rescale(e.upload(a, mid), e.upload(b, mid), rk)
                        .download())
    finally:
        lib.fhe_ntt_tuning_set(log_n, *saved)
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
