"""The two forms of the base conversions give the same words: the INT8 tensor-core
forms (tcgen05.mma kind::i8; ModDown's division by the special primes and ModUp's
digit contraction) and the CUDA-core forms (the reference's operation order),
on every key-switching operation, several levels and three parameter sets.  The
recorded-reference and oracle parity suites run the tensor-core form too."""
import numpy as np
import pytest

from inputs import uniform_limbs

pytestmark = pytest.mark.gpu

NTT, RESCALED, SPECIAL = 2, 4, 16
RELIN, FIXED_ROTATION, KEY_SWITCHING = 3, 6, 8

CONFIGS = [  # (log_n, special primes, preset, moduli ids)
    (16, 10, 1, [1, 5, 12]),
    (16, 4, 2, [2, 9, 20]),
    (14, 1, 1, [1, 4]),
    (15, 2, 1, [1, 7]),
    (17, 6, 1, [1]),
]


def run_both(e, fn):
    """fn() with the tensor-core form, then with the CUDA-core form."""
    e.set_tensor_cores(True)
    e.set_profiling(True)
    e.profile_reset()
    tc = fn()
    families = e.profile()
    e.set_tensor_cores(False)
    try:
        plain = fn()
    finally:
        e.set_tensor_cores(2)
        e.set_profiling(False)
    return tc, plain, families


@pytest.mark.parametrize("log_n,K,preset,mids", CONFIGS, ids=lambda v: str(v))
def test_tensor_core_mod_down_matches_cuda_core(engines, log_n, K, preset, mids):
    e = engines(log_n, K, preset)
    n = e.coeff_count
    for mid in mids:
        rng = np.random.default_rng(9000 + 100 * log_n + 10 * K + mid)
        a = uniform_limbs(rng, e.moduli[mid:e.chain_count], 2, n)
        b = uniform_limbs(rng, e.moduli[mid:e.chain_count], 2, n)
        t3 = uniform_limbs(rng, e.moduli[mid:e.chain_count], 3, n)
        key = uniform_limbs(rng, e.moduli[mid:], 2 * e.partition_count(mid), n)
        rk = e.upload(key, mid, NTT | SPECIAL, RELIN)
        fk = e.upload_fixed_rotation_key(key, mid, 3)
        ksk = e.upload_key_switching_key(key, mid)

        def ops():
            out = [e.relinearize(e.upload(t3, mid, NTT), rk).download(),
                   e.rotate(e.upload(a, mid), fk).download(),
                   e.switch_key(e.upload(b, mid), ksk).download()]
            if e.chain_count - mid >= 3:
                out.append(e.multiply_relinearize_rescale(e.upload(a, mid, NTT),
                                                          e.upload(b, mid, NTT), rk).download())
            return out

        tc, plain, families = run_both(e, ops)
        assert "mod_down_epilogue_tc" in families, families
        assert "mod_down_epilogue" not in families, families
        assert "mod_up_ntt_tc" in families, families
        assert "mod_up_ntt" not in families, families
        for got, want in zip(tc, plain):
            assert np.array_equal(got, want)
