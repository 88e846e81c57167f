"""GPU parity of bootstrapping: the bootstrap preset at N = 2^16 with 4 special
primes and 3 stages, keys made on the device from the reseeded random stream, then
bootstrap(ct, rk, ck, rotation key, small bootstrap key) through the C ABI.  Every
key and the bootstrapped ciphertext must equal the reference's words; the decoded
slots keep the reference's ~18 bits of precision."""
import numpy as np
import pytest

from conftest import load_golden
from inputs import codec_values, digest, digest_doubles

pytestmark = pytest.mark.gpu

CASES = load_golden("bootstrap.json")


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["tier"])
def test_bootstrap_matches_recorded_reference(engines, case):
    e = engines(case["log_n"], case["special_prime_count"], case["preset"])
    assert e.moduli.tolist() == case["moduli"]
    d = case["digests"]
    e.seed(case["seed"], case["nonce"])
    sk = e.create_secret_key()
    assert digest(sk.download()) == d["secret_key"]
    rk = e.create_relinearization_key(sk)
    assert digest(rk.download()) == d["relinearization_key"]
    ck = e.create_conjugation_key(sk)
    assert digest(ck.download()) == d["conjugation_key"]
    rot = e.create_rotation_key(sk)
    assert [k.info()["delta"] for k in rot] == case["rotation_deltas"]
    assert digest(rot[0].download()) == d["rotation_key_1"]
    assert [digest(k.download()) for k in rot] == case["rotation_keys"]
    to_sparse, to_dense = e.create_small_bootstrap_key(sk)
    assert digest(to_sparse.download()) == d["to_sparse"]
    assert digest(to_dense.download()) == d["to_dense"]
    vals = codec_values(case["values_seed"], e.slot_count, True)
    ct = e.encrypt(e.encode(vals, case["encrypt_level"]), sk)
    assert digest(ct.download()) == d["ciphertext"]
    out = e.bootstrap(ct, rk, ck, rot, (to_sparse, to_dense), case["stage_count"])
    info = out.info()
    assert (info["moduli_id"], info["level"]) == (case["output_moduli_id"], case["output_level"])
    assert digest(out.download()) == d["bootstrapped"]
    slots = e.decode(e.decrypt(out, sk), complex_output=True)
    assert digest_doubles(slots) == case["decoded"]
    assert np.max(np.abs(slots - vals)) < 2.0 ** -16
