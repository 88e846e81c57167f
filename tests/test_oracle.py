"""Pin the CPU oracle: the reference's own known-answer tests, recorded reference
outputs on seeded inputs, and (where it is built) the reference library itself."""
import os

import numpy as np
import pytest

from conftest import load_golden
from inputs import ROTATION_KEY_DELTAS, codec_values, digest_doubles, key_switch_inputs, TIERS, case_inputs, digest
from oracle import oracle, ref


@pytest.mark.parametrize("kat", load_golden("ntt_kat.json"), ids=lambda k: k["name"])
def test_ntt_known_answers(kat):
    """test/operation/ntt.cpp: N=16 transforms with explicit roots."""
    x = np.array(kat["x"], dtype=np.int64)
    table = np.array(kat["table"], dtype=np.int64)
    if kat["kind"] == "ntt":
        y = oracle.ntt_limb(x, table, kat["q"], kat["k"])
    else:
        y = oracle.intt_limb(x, table, kat["q"], kat["k"])
    assert y.tolist() == kat["expected"]


def test_montgomery_scalar_known_answers():
    """test/montgomery/unit.cpp: Multiply / MultiplyR and the k of q=1099516280833."""
    q, k = 1099516280833, 2888757134567604223
    assert oracle.calculate_k(q) == k
    assert [oracle.mont_mult(a, 2, q, k) for a in (1, 2)] == [277956291297, 555912582594]
    r = 1 << 62
    assert [oracle.mont_mult(a, r, q, k) for a in (1, 2)] == [1, 2]


def _kat_items():
    out = []
    for name, entry in load_golden("precomputed_kat.json").items():
        out.append((name, entry))
    return out


@pytest.mark.parametrize("name,entry", _kat_items(), ids=[n for n, _ in _kat_items()])
def test_oracle_tables_match_precomputed_known_answers(name, entry):
    """test/ckks/precomputed/default.cpp: chains, k, r^2, N^-1, roots per tier."""
    log_n, K, preset = TIERS[entry["tier"]]
    v = entry["vectors"]
    q = np.array(v["q"], dtype=np.uint64)
    if log_n > 14:
        pytest.skip("large tiers are covered through the product parameter test")
    ctx = oracle.Context(log_n, q, K)
    t = ctx.tables()
    n = 1 << log_n
    assert t["k"][: len(v["k"])].tolist() == v["k"]
    assert t["r_squared"][: len(v["r_squared"])].tolist() == v["r_squared"]
    assert t["n_inverse"][: len(v["coeff_count_inverse"])].tolist() == v["coeff_count_inverse"]
    assert t["root"].reshape(-1)[: len(v["root"])].tolist() == v["root"]
    assert t["root_inverse"].reshape(-1)[: len(v["root_inverse"])].tolist() == v["root_inverse"]
    assert n == 1 << log_n


def _cases():
    return [c for c in load_golden("ref_ops.json") if c["log_n"] <= 14]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: f"{c['tier']}-m{c['moduli_id']}")
def test_oracle_matches_recorded_reference_outputs(case):
    """Oracle vs outputs recorded from the compiled reference on the same inputs."""
    log_n, K = case["log_n"], case["special_prime_count"]
    q = _chain(case)
    ctx = oracle.Context(log_n, q, K)
    mid = case["moduli_id"]
    a, b, ct3, key = case_inputs(case["seed"], q, ctx.n, mid, K)
    got = {
        "to_ntt": ctx.to_ntt(mid, a),
        "to_intt": ctx.to_intt(mid, a),
        "tensor": ctx.tensor(mid, a, b),
        "relinearize": ctx.relinearize(mid, ct3, mid, key),
        "rescale": ctx.rescale(mid, a),
    }
    if "mult_relin_rescale" in case["digests"]:
        got["mult_relin_rescale"] = ctx.mult_relin_rescale(mid, a, b, mid, key)
    for name, arr in got.items():
        assert digest(arr) == case["digests"][name], name


@pytest.mark.parametrize("case", load_golden("ref_ops_c10.json"), ids=lambda c: f"c10-m{c['moduli_id']}")
def test_oracle_matches_reference_at_headline_config(case):
    """Oracle vs the compiled reference at N = 2^16 with 10 special primes (dnum = 3,
    partitions of up to 10 limbs): relinearization and the fused multiply chain."""
    q = _chain(case)
    ctx = oracle.Context(case["log_n"], q, case["special_prime_count"])
    mid = case["moduli_id"]
    a, b, ct3, key = case_inputs(case["seed"], q, ctx.n, mid, case["special_prime_count"])
    assert digest(ctx.relinearize(mid, ct3, mid, key)) == case["digests"]["relinearize"]
    assert digest(ctx.mult_relin_rescale(mid, a, b, mid, key)) == case["digests"]["mult_relin_rescale"]


def _chain(case):
    return np.array(case["moduli"], dtype=np.uint64)


def _engine_scale(case):
    return 2.0 ** (54 if case["preset"] in (2, 4) else 40)


def _switch_input(ctx, case, mid, x, ntt):
    """The engine's preparation of a rotation/conjugation input (engine_rotate.cpp:52-74):
    a text at moduli id 0 drops one level first (one-more-level rule), then leaves NTT form."""
    if mid == 0:
        level = ctx.chains(0) - 2
        y = ctx.to_intt(0, x) if ntt else x
        y = ctx.level_down(y, level, level - 1, False, _engine_scale(case), True)
        if ntt:
            y = ctx.to_ntt(1, y)
        return 1, (ctx.to_intt(1, y) if ntt else y)
    return mid, (ctx.to_intt(mid, x) if ntt else x)


@pytest.mark.parametrize("case", _cases(), ids=lambda c: f"{c['tier']}-m{c['moduli_id']}")
def test_oracle_key_switch_ops_match_recorded_reference(case):
    """Rotation, conjugation, switch_key, keyless rotations, level down and a
    mixed-level multiply composed from oracle steps, against the reference's engine."""
    log_n, K = case["log_n"], case["special_prime_count"]
    q = _chain(case)
    ctx = oracle.Context(log_n, q, K)
    mid, n = case["moduli_id"], ctx.n
    a, _, _, key = case_inputs(case["seed"], q, n, mid, K)
    x = key_switch_inputs(case["seed"], q, n, mid, K)
    kmid, keys = x["key_moduli_id"], x["rotation_keys"]
    d = case["digests"]
    scale = _engine_scale(case)

    def rotate(m, y, i):
        return ctx.rotate(m, y, kmid, keys[i], ROTATION_KEY_DELTAS[i])

    m, y = _switch_input(ctx, case, mid, a, False)
    assert digest(rotate(m, y, 0)) == d["rotate_1"]
    m4, y4 = _switch_input(ctx, case, mid, a, True)
    assert digest(rotate(m4, y4, 2)) == d["rotate_4_ntt"]
    nd, cur, cm = 7 % (n // 2), a, mid
    for i, delta in enumerate(ROTATION_KEY_DELTAS):
        if nd & delta:
            cm, cur = _switch_input(ctx, case, cm, cur, False)
            cur = rotate(cm, cur, i)
    assert digest(cur) == d["rotate_keys_7"]
    assert digest(ctx.conjugate(m, y, kmid, x["conjugation_key"])) == d["conjugate"]
    assert digest(ctx.switch_key(mid, a, mid, x["switching_key"])) == d["switch_key"]
    p = a[:1]
    assert digest(ctx.rotate_plain(mid, p, 3 % (n // 2))) == d["rotate_plain_3"]
    assert digest(ctx.rotate_plain(mid, p, 3 % (n // 2), True)) == d["rotate_plain_3_ntt"]
    assert digest(ctx.rotate_plain(mid, p, -1)) == d["conjugate_plain"]
    assert digest(ctx.rotate_plain(mid, p, -1, True)) == d["conjugate_plain_ntt"]
    level = ctx.chains(mid) - 2
    full = ctx.chain_count - 2
    if "level_down" in d:
        assert digest(ctx.level_down(a, level, level - 1, False, scale, True)) == d["level_down"]
        down = ctx.level_down(ctx.to_intt(mid, a), level, 0, False, scale, True)
        assert digest(ctx.to_ntt(full, down)) == d["level_down_ntt"]
    if "level_down_rescaled" in d:
        got = ctx.level_down(a, level + 1, level, True, scale, True)
        assert digest(got) == d["level_down_rescaled"]
    if "multiply_mixed_levels" in d:
        la = ctx.level_down(a, level, level - 1, False, scale, True)
        na = ctx.to_ntt(mid + 2, ctx.rescale(mid + 1, la))
        nb = ctx.to_ntt(mid + 2, ctx.rescale(mid + 1, x["b_next"]))
        got = ctx.relinearize(mid + 2, ctx.tensor(mid + 2, na, nb), mid, key)
        assert digest(got) == d["multiply_mixed_levels"]


@pytest.mark.skipif(not ref.available(), reason="reference library not built")
@pytest.mark.parametrize("tier,mid", [("pebble", 0), ("bronze", 2), ("silver", 3)])
def test_oracle_matches_live_reference(tier, mid):
    log_n, K, preset = TIERS[tier]
    e = ref.Engine(log_n=log_n, special_prime_count=K, preset=preset)
    q = e.tables()["q"]
    ctx = oracle.Context(log_n, q, K)
    a, b, ct3, key = case_inputs(77 + mid, q, e.n, mid, K)
    rk = e.relin_key(key, mid)
    r = e.core_relinearize(e.text(ct3, mid, flag=2), rk).limbs()
    assert np.array_equal(r, ctx.relinearize(mid, ct3, mid, key))
    m = e.rescale(e.multiply(e.text(a, mid, flag=0), e.text(b, mid, flag=0), rk)).limbs()
    assert np.array_equal(m, ctx.mult_relin_rescale(mid, a, b, mid, key))


@pytest.mark.parametrize("n,delta", [(16, 1), (16, 3), (16, -1), (64, 5), (1024, 7), (1024, -1)])
def test_rotation_permutations_are_permutations(n, delta):
    perm, sign = oracle.permutation_and_sign(n, delta)
    assert sorted(perm.tolist()) == list(range(n))
    assert set(sign.tolist()) <= {-1, 1}
    nperm = oracle.ntt_permutation(n, delta)
    assert sorted(nperm.tolist()) == list(range(n))


@pytest.mark.parametrize("case", load_golden("codec.json"),
                         ids=lambda c: f"{c['tier']}-s{c['log_slot']}-l{c['level']}-{c['kind']}")
def test_oracle_codec_matches_recorded_reference(case):
    """Encode limbs and decoded doubles (bit patterns) of the oracle's restatement
    against the reference's encode_unit / decode_unit on the same slot values."""
    log_n, K = case["log_n"], case["special_prime_count"]
    ctx = oracle.Context(log_n, _chain(case), K)
    log_slot = log_n - 1 if case["log_slot"] < 0 else case["log_slot"]
    complex_values = case["kind"] == "complex"
    vals = codec_values(case["seed"], 1 << log_slot, complex_values)
    limbs, ckks_scale = ctx.encode(vals, log_slot, case["level"], case["scale_bits"])
    assert digest(limbs) == case["encode"]
    dec = ctx.decode_plaintext(limbs[0], case["moduli_id"], log_slot, ckks_scale,
                               case["scale_bits"], complex_output=complex_values)
    assert digest_doubles(dec) == case["decode"]


def test_oracle_random_stream_matches_known_answers():
    """test/random/random.cpp: ChaCha20 blocks 0-3, rand_int (max 10, shift 0 and 10)
    and discrete_gaussian outputs of the test state."""
    kat = load_golden("random_kat.json")
    seed, nonce = kat["seed"], kat["nonce"]
    for counter, block in enumerate(kat["chacha20"]):
        assert oracle.chacha_block(seed, nonce, counter) == block
    assert oracle.rand_int(seed, nonce, 0, 32, 10).tolist() == kat["rand_int_10"]
    assert oracle.rand_int(seed, nonce, 0, 32, 10, 10).tolist() == kat["rand_int_10_shift_10"]
    got = oracle.discrete_gaussian(seed, nonce, 0, 32, kat["cdt_tree"])
    assert got.tolist() == kat["discrete_gaussian"]


def test_engine_cdt_table_is_the_reference_tree():
    """fhe_b200/csrc/cdt_table.inc holds the tree literal of gaussian_sampler.cpp."""
    import re

    text = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                             "fhe_b200", "csrc", "cdt_table.inc")).read()
    words = [int(w) for w in re.findall(r"(\d+)ULL", text)]
    assert words == load_golden("random_kat.json")["cdt_tree"]
