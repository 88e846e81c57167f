"""GPU parity of encode and decode: the device FFT, twist, rounding and CRT
reconstruction against the reference's encode_unit / decode_unit on the same slot
values.  Limbs are compared word for word and decoded slots by their IEEE bit
patterns (the device performs the reference's double operations in its order)."""
import numpy as np
import pytest

from conftest import load_golden
from inputs import codec_values, digest, digest_doubles

pytestmark = pytest.mark.gpu

CASES = load_golden("codec.json")


@pytest.mark.parametrize("case", CASES,
                         ids=lambda c: f"{c['tier']}-s{c['log_slot']}-l{c['level']}-{c['kind']}")
def test_codec_matches_recorded_reference(engines, case):
    e = engines(case["log_n"], case["special_prime_count"], case["preset"], case["log_slot"])
    assert e.moduli.tolist() == case["moduli"]
    complex_values = case["kind"] == "complex"
    vals = codec_values(case["seed"], e.slot_count, complex_values)
    pt = e.encode(vals, case["level"])
    assert pt.info()["moduli_id"] == case["moduli_id"]
    assert digest(pt.download()) == case["encode"]
    dec = e.decode(pt, complex_output=complex_values)
    assert digest_doubles(dec) == case["decode"]
    assert np.max(np.abs(dec - vals)) == pytest.approx(case["max_error"], rel=0, abs=0)


def test_decode_rejects_rescaled_plaintexts(engines):
    from fhe_b200 import FheError, RESCALED, UNIT_PLAINTEXT

    e = engines(14, 1, 1)
    limbs = np.zeros((1, e.chains(2), e.coeff_count), dtype=np.int64)
    pt = e.upload(limbs, 2, RESCALED, UNIT_PLAINTEXT)
    with pytest.raises(FheError, match="should not be rescaled"):
        e.decode(pt)


def test_encode_pads_short_inputs_with_zeros(engines):
    e = engines(14, 1, 1)
    short = np.linspace(-1, 1, 100)
    padded = np.zeros(e.slot_count)
    padded[:100] = short
    a = e.encode(short, 3).download()
    b = e.encode(padded, 3).download()
    assert np.array_equal(a, b)
