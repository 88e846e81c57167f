"""Pin the CPU oracle: the reference's own known-answer tests, recorded reference
outputs on seeded inputs, and (where it is built) the reference library itself."""
import numpy as np
import pytest

from conftest import load_golden
from inputs import TIERS, case_inputs, digest
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


def _chain(case):
    return np.array(case["moduli"], dtype=np.uint64)


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
