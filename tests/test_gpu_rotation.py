"""GPU parity of rotation, conjugation, key switching and level down: the sm_100a
path through the C ABI against the recorded reference outputs (every tier) and the
CPU oracle at N = 2^16 with 10 special primes.  All bit-exact."""
import numpy as np
import pytest

from conftest import load_golden
from inputs import ROTATION_KEY_DELTAS, case_inputs, digest, key_switch_inputs, uniform_limbs
from oracle import oracle

pytestmark = pytest.mark.gpu

NTT, RESCALED, SPECIAL = 2, 4, 16
SCALE = 2.0 ** 40

CASES = [c for c in load_golden("ref_ops.json") if "rotate_1" in c["digests"]]


HEADLINE_CASES = load_golden("ref_ops_c10.json")


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c['tier']}-m{c['moduli_id']}")
def test_key_switch_ops_match_recorded_reference(engines, case):
    check_key_switch_ops(engines(case["log_n"], case["special_prime_count"], case["preset"]), case)


@pytest.mark.parametrize("mode", [1, 0], ids=["tensor-cores", "cuda-cores"])
@pytest.mark.parametrize("case", HEADLINE_CASES, ids=lambda c: f"{c['tier']}-m{c['moduli_id']}")
def test_headline_key_switch_ops_match_recorded_reference(engines, case, mode):
    """Rotations, conjugation, key switching, level down and the mixed-level multiply
    at N = 2^16 with 10 special primes, against the reference's own words, with the
    base conversions on the tensor pipe and then on the CUDA cores."""
    e = engines(case["log_n"], case["special_prime_count"], case["preset"])
    e.set_tensor_cores(mode)
    try:
        check_key_switch_ops(e, case)
    finally:
        e.set_tensor_cores(2)


def check_key_switch_ops(e, case):
    from fhe_b200 import RELINEARIZATION_KEY, UNIT_PLAINTEXT

    q = np.array(case["moduli"], dtype=np.uint64)
    assert e.moduli.tolist() == case["moduli"]
    mid, K, n = case["moduli_id"], case["special_prime_count"], e.coeff_count
    a, _, _, key = case_inputs(case["seed"], q, n, mid, K)
    x = key_switch_inputs(case["seed"], q, n, mid, K)
    kmid = x["key_moduli_id"]
    fks = [e.upload_fixed_rotation_key(k, kmid, d)
           for k, d in zip(x["rotation_keys"], ROTATION_KEY_DELTAS)]
    ck = e.upload_conjugation_key(x["conjugation_key"], kmid)
    d = case["digests"]

    def ct(flag=0):
        return e.upload(a, mid, flag, scale=SCALE)

    assert digest(e.rotate(ct(), fks[0]).download()) == d["rotate_1"]
    assert digest(e.rotate(ct(NTT), fks[2]).download()) == d["rotate_4_ntt"]
    assert digest(e.rotate(ct(), fks, 7).download()) == d["rotate_keys_7"]
    assert digest(e.conjugate(ct(), ck).download()) == d["conjugate"]
    ksk = e.upload_key_switching_key(x["switching_key"], mid)
    assert digest(e.switch_key(ct(), ksk).download()) == d["switch_key"]

    def pt(flag):
        return e.upload(a[:1], mid, flag, UNIT_PLAINTEXT)

    assert digest(e.rotate_plaintext(pt(0), 3).download()) == d["rotate_plain_3"]
    assert digest(e.rotate_plaintext(pt(NTT), 3).download()) == d["rotate_plain_3_ntt"]
    assert digest(e.conjugate(pt(0)).download()) == d["conjugate_plain"]
    assert digest(e.conjugate(pt(NTT)).download()) == d["conjugate_plain_ntt"]

    level = e.chains(mid) - 2
    if "level_down" in d:
        assert digest(e.level_down(ct(), level - 1).download()) == d["level_down"]
        assert digest(e.level_down(ct(NTT), 0).download()) == d["level_down_ntt"]
    if "level_down_rescaled" in d:
        assert digest(e.level_down(ct(RESCALED), level).download()) == d["level_down_rescaled"]
    if "multiply_mixed_levels" in d:
        rk = e.upload(key, mid, NTT | SPECIAL, RELINEARIZATION_KEY)
        b_next = e.upload(x["b_next"], mid + 1, scale=SCALE)
        assert digest(e.multiply(ct(), b_next, rk).download()) == d["multiply_mixed_levels"]


@pytest.fixture(scope="module")
def config_c(engines):
    e = engines(16, 10, 1)
    return e, oracle.Context(16, e.moduli, 10)


@pytest.mark.parametrize("delta", [1, 5, 1 << 14])
def test_full_size_rotate_matches_oracle(config_c, delta):
    e, ctx = config_c
    mid = e.moduli_id(e.max_key_switching_level)
    rng = np.random.default_rng(7000 + delta)
    a = uniform_limbs(rng, e.moduli[mid:e.chain_count], 2, e.coeff_count)
    key = uniform_limbs(rng, e.moduli[mid:], 2 * e.partition_count(mid), e.coeff_count)
    fk = e.upload_fixed_rotation_key(key, mid, delta)
    got = e.rotate(e.upload(a, mid), fk).download()
    assert np.array_equal(got, ctx.rotate(mid, a, mid, key, delta))


def test_full_size_conjugate_and_switch_key_match_oracle(config_c):
    e, ctx = config_c
    mid, key_mid = 3, 1
    rng = np.random.default_rng(7100)
    a = uniform_limbs(rng, e.moduli[mid:e.chain_count], 2, e.coeff_count)
    key = uniform_limbs(rng, e.moduli[key_mid:], 2 * e.partition_count(key_mid), e.coeff_count)
    got = e.conjugate(e.upload(a, mid), e.upload_conjugation_key(key, key_mid)).download()
    assert np.array_equal(got, ctx.conjugate(mid, a, key_mid, key))
    got = e.switch_key(e.upload(a, mid), e.upload_key_switching_key(key, key_mid)).download()
    assert np.array_equal(got, ctx.switch_key(mid, a, key_mid, key))


def test_rotation_round_trip_by_composition(config_c):
    """Rotating by keys for deltas 1, 2 and 4 with delta 7 equals applying the three
    fixed rotations one after another (the reference's loop, engine_rotate.cpp:126-137)."""
    e, _ = config_c
    mid = 4
    rng = np.random.default_rng(7200)
    a = e.upload(uniform_limbs(rng, e.moduli[mid:e.chain_count], 2, e.coeff_count), mid)
    keys = [e.upload_fixed_rotation_key(
        uniform_limbs(rng, e.moduli[mid:], 2 * e.partition_count(mid), e.coeff_count), mid, dd)
        for dd in (1, 2, 4)]
    combined = e.rotate(a, keys, 7).download()
    step = a
    for k in keys:
        step = e.rotate(step, k)
    assert np.array_equal(combined, step.download())


def test_rotation_errors_mirror_reference(config_c):
    from fhe_b200 import FheError

    e, _ = config_c
    rng = np.random.default_rng(7300)
    a = e.upload(uniform_limbs(rng, e.moduli[5:e.chain_count], 2, e.coeff_count), 5)
    key = uniform_limbs(rng, e.moduli[6:], 2 * e.partition_count(6), e.coeff_count)
    fk = e.upload_fixed_rotation_key(key, 6, 1)
    with pytest.raises(FheError, match="greater than that of the input fixed rotation key"):
        e.rotate(a, fk)
    with pytest.raises(FheError, match="target level cannot be reached"):
        e.level_down(a, 40)


@pytest.mark.parametrize("mid,key_mid", [(1, 1), (6, 1), (12, 3)])
def test_hoisted_rotate_batch_matches_single_rotations(config_c, mid, key_mid):
    """rotate_batch with fixed keys (one decomposition, engine_rotate.cpp:262-300)
    gives the words of one rotation per key, for keys at the text's level or above."""
    e, _ = config_c
    rng = np.random.default_rng(7300 + mid)
    a = e.upload(uniform_limbs(rng, e.moduli[mid:e.chain_count], 2, e.coeff_count), mid)
    keys = [e.upload_fixed_rotation_key(
        uniform_limbs(rng, e.moduli[key_mid:], 2 * e.partition_count(key_mid), e.coeff_count),
        key_mid, d) for d in (1, 3, 1 << 10)]
    hoisted = e.rotate_batch(a, keys)
    for k, h in zip(keys, hoisted):
        assert np.array_equal(h.download(), e.rotate(a, k).download())

