"""GPU parity of randomness, key generation, encryption and decryption: the
engine's ChaCha20 stream reseeded like the reference's, then the same sequence of
calls (secret key, public key, relinearization, rotation and conjugation keys,
public- and secret-key encryption, decryption, decode) must give the reference's
words exactly."""
import numpy as np
import pytest

from conftest import load_golden
from inputs import codec_values, digest, digest_doubles

pytestmark = pytest.mark.gpu

CASES = load_golden("keygen.json")


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["tier"])
def test_keys_and_encryption_match_recorded_reference(engines, case):
    e = engines(case["log_n"], case["special_prime_count"], case["preset"])
    assert e.moduli.tolist() == case["moduli"]
    d = case["digests"]
    e.seed(case["seed"], case["nonce"])
    sk = e.create_secret_key()
    assert digest(sk.download()) == d["secret_key"]
    pk = e.create_public_key(sk)
    assert digest(pk.download()) == d["public_key"]
    rk = e.create_relinearization_key(sk)
    assert digest(rk.download()) == d["relinearization_key"]
    fk = e.create_fixed_rotation_key(sk, 3)
    assert digest(fk.download()) == d["fixed_rotation_key_3"]
    ck = e.create_conjugation_key(sk)
    assert digest(ck.download()) == d["conjugation_key"]
    vals = codec_values(case["values_seed"], e.slot_count, True)
    pt = e.encode(vals, case["level"])
    assert digest(pt.download()) == d["plaintext"]
    ct_pk = e.encrypt(pt, pk)
    assert digest(ct_pk.download()) == d["encrypt_public"]
    ct_sk = e.encrypt(pt, sk)
    assert digest(ct_sk.download()) == d["encrypt_secret"]
    dec = e.decrypt(ct_pk, sk)
    assert digest(dec.download()) == d["decrypt_public"]
    slots = e.decode(dec, complex_output=True)
    assert digest_doubles(slots) == case["decoded"]


def test_encrypt_multiply_decrypt_round_trip(engines):
    """Plain CKKS at N = 2^14 (the reference's default engine): encode two vectors,
    encrypt, multiply with relinearization, rescale, decrypt, decode; slots within
    2^-20 of the float64 elementwise product."""
    e = engines(14, 1, 1)
    e.seed(list(range(1, 9)), [3, 4])
    sk = e.create_secret_key()
    pk = e.create_public_key(sk)
    rk = e.create_relinearization_key(sk)
    rng = np.random.default_rng(2024)
    n = e.slot_count
    a = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    b = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    level = e.max_key_switching_level
    ca = e.encrypt(e.encode(a, level), pk)
    cb = e.encrypt(e.encode(b, level), pk)
    prod = e.rescale(e.multiply(ca, cb, rk))
    out = e.decode(e.decrypt(prod, sk), complex_output=True)
    err = np.max(np.abs(out - a * b))
    assert err < 2.0 ** -20, err


def test_serialized_objects_round_trip(engines):
    """Keys and ciphertexts survive the wire format word for word, with their
    metadata; an engine with other parameters or a damaged header rejects them."""
    from fhe_b200._lib import FheError

    e = engines(14, 1, 1)
    sk = e.create_secret_key()
    rk = e.create_relinearization_key(sk)
    ct = e.encrypt(e.encode(np.linspace(-1, 1, e.slot_count)), sk)
    for obj in (sk, rk, ct):
        blob = obj.serialize()
        back = e.deserialize(blob)
        assert back.info() == obj.info()
        assert np.array_equal(back.download(), obj.download())
    blob = bytearray(ct.serialize())
    with pytest.raises(FheError, match="deserialize"):
        engines(15, 2, 1).deserialize(bytes(blob))
    blob[0:8] = b"NOTADATA"
    with pytest.raises(FheError, match="not a serialized engine object"):
        e.deserialize(bytes(blob))

