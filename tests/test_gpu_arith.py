"""GPU parity of ciphertext arithmetic: additions, subtractions, plaintext and
scalar products, negation and squaring through the C ABI, against the reference's
engine on the same operands (level matching, rescale state and NTT form included)."""
import pytest

from conftest import load_golden
from inputs import arith_inputs, digest

pytestmark = pytest.mark.gpu

CASES = load_golden("arith.json")
SCALAR_OPS = {"add_scalar", "subtract_scalar", "multiply_scalar", "multiply_integer"}


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c['tier']}-m{c['moduli_id']}")
def test_arithmetic_matches_recorded_reference(engines, case):
    from fhe_b200 import NTT_FORM, INCLUDE_SPECIAL, RELINEARIZATION_KEY, UNIT_CIPHERTEXT, UNIT_PLAINTEXT

    e = engines(case["log_n"], case["special_prime_count"], case["preset"])
    assert e.moduli.tolist() == case["moduli"]
    mid = case["moduli_id"]
    x = arith_inputs(case["seed"], e.moduli, e.coeff_count, mid, case["special_prime_count"])
    rk = e.upload(x["key"], mid, NTT_FORM | INCLUDE_SPECIAL, RELINEARIZATION_KEY)

    def text(spec):
        name, flag = spec.split(":")
        m = mid + 1 if name == "low" else mid
        kind = UNIT_PLAINTEXT if name == "plain" else UNIT_CIPHERTEXT
        scale = case["low_scale"] if name == "low" else case["scale"]
        return e.upload(x[name], m, int(flag), kind, scale)

    failures = []
    for key, want in case["digests"].items():
        step = key.split("|")
        op = step[0]
        if op in SCALAR_OPS:
            value = int(step[2]) if op == "multiply_integer" else float(step[2])
            a = text(step[1])
            out = {"add_scalar": lambda: e.add(a, value),
                   "subtract_scalar": lambda: e.subtract(a, value),
                   "multiply_scalar": lambda: e.multiply_scalar(a, value),
                   "multiply_integer": lambda: e.multiply_integer(a, value)}[op]()
        elif op == "negate":
            out = e.negate(text(step[1]))
        elif op == "square":
            out = e.square(text(step[1]))
        elif op == "square_relinearize":
            out = e.square(text(step[1]), rk)
        elif op == "subtract_from_plain":
            out = e.subtract(text(step[2]), text(step[1]))
        elif op == "multiply_plain":
            out = e.multiply_plaintext(text(step[1]), text(step[2]))
        elif op in ("add", "add_plain"):
            out = e.add(text(step[1]), text(step[2]))
        else:
            out = e.subtract(text(step[1]), text(step[2]))
        if digest(out.download()) != want:
            failures.append(key)
    assert not failures, failures
