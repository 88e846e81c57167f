"""GPU parity of the plain CKKS pipeline (the reference's default engine, N = 2^14 with
one special prime, and the gold tier): keys from the reseeded random stream, two
complex vectors encoded and encrypted with the public key, multiplied with the
relinearization key, rescaled, decrypted and decoded.  Every ciphertext's words
and the decoded slots equal the reference's; the slots match the float64 product."""
import numpy as np
import pytest

from conftest import load_golden
from inputs import codec_values, digest, digest_doubles

pytestmark = pytest.mark.gpu

CASES = load_golden("pipeline.json")


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["tier"])
def test_pipeline_matches_recorded_reference(engines, case):
    e = engines(case["log_n"], case["special_prime_count"], case["preset"])
    assert e.moduli.tolist() == case["moduli"]
    d = case["digests"]
    e.seed(case["seed"], case["nonce"])
    sk = e.create_secret_key()
    pk = e.create_public_key(sk)
    rk = e.create_relinearization_key(sk)
    assert digest(pk.download()) == d["public_key"]
    va = codec_values(case["values_seeds"][0], e.slot_count, True)
    vb = codec_values(case["values_seeds"][1], e.slot_count, True)
    a = e.encrypt(e.encode(va), pk)
    b = e.encrypt(e.encode(vb), pk)
    assert digest(a.download()) == d["ct_a"]
    assert digest(b.download()) == d["ct_b"]
    product = e.multiply(a, b, rk)
    assert digest(product.download()) == d["product"]
    rescaled = e.rescale(product)
    info = rescaled.info()
    assert (info["moduli_id"], info["level"]) == (case["rescaled_moduli_id"], case["rescaled_level"])
    assert digest(rescaled.download()) == d["rescaled"]
    slots = e.decode(e.decrypt(rescaled, sk), complex_output=True)
    assert digest_doubles(slots) == case["decoded"]
    assert np.max(np.abs(slots - va * vb)) <= case["max_error"]
    assert np.max(np.abs(slots - va * vb)) < 2.0 ** -20
