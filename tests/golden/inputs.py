"""Seeded synthetic inputs shared by the fixture generator and the tests.

Residues are uniform in [0, q_i) per limb from numpy's PCG64 generator, so a
fixture only needs to store its seed and the digest of the expected output.
"""
from __future__ import annotations

import hashlib

import numpy as np

# (log_n, special_prime_count, scheme_preset) of the reference's tiers
# (ckks/config.cpp:106-139, for_bootstrap :188-193).  Sand/Pebble use the
# engine-test preset, which has the same chain as the default preset there.
TIERS = {
    "sand": (3, 1, 3),
    "pebble": (4, 1, 3),
    "iron": (13, 1, 1),
    "bronze": (14, 1, 1),
    "silver": (15, 2, 1),
    "gold": (16, 4, 1),
    "c10": (16, 10, 1),  # the headline key-switching set: 10 special primes, dnum = 3
    "platinum": (17, 6, 1),
    "bootstrap_gold": (16, 4, 2),
}


def uniform_limbs(rng: np.random.Generator, moduli, polys: int, n: int) -> np.ndarray:
    out = np.empty((polys, len(moduli), n), dtype=np.int64)
    for p in range(polys):
        for j, q in enumerate(moduli):
            out[p, j] = rng.integers(0, int(q), size=n, dtype=np.int64)
    return out


def digest(a: np.ndarray) -> str:
    a = np.ascontiguousarray(a, dtype=np.int64)
    return hashlib.sha256(a.tobytes()).hexdigest()


def case_inputs(seed: int, moduli, n: int, moduli_id: int, special: int):
    """Inputs of one op-parity case at `moduli_id`: two 2-poly texts, one 3-poly
    NTT text and a relinearization key at the same moduli id."""
    rng = np.random.default_rng(seed)
    chain = len(moduli) - special
    L = chain - moduli_id
    qs = moduli[moduli_id:moduli_id + L]
    ext = moduli[moduli_id:]
    dnum = (L + special - 1) // special
    a = uniform_limbs(rng, qs, 2, n)
    b = uniform_limbs(rng, qs, 2, n)
    ct3 = uniform_limbs(rng, qs, 3, n)
    key = uniform_limbs(rng, ext, 2 * dnum, n)
    return a, b, ct3, key


ROTATION_KEY_DELTAS = (1, 2, 4)


def key_switch_inputs(seed: int, moduli, n: int, moduli_id: int, special: int):
    """Inputs of the rotation / conjugation / key-switch / level cases of one
    op-parity case, drawn from their own stream so the other inputs keep their
    values.  Texts at moduli id 0 are switched at moduli id 1 by the engine (the
    one-more-level rule), so their rotation and conjugation keys live there."""
    rng = np.random.default_rng(seed + 100000)
    chain = len(moduli) - special

    def key_at(mid):
        dnum = (chain - mid + special - 1) // special
        return uniform_limbs(rng, moduli[mid:], 2 * dnum, n)

    key_mid = moduli_id if moduli_id > 0 else 1
    rotation_keys = [key_at(key_mid) for _ in ROTATION_KEY_DELTAS]
    conjugation_key = key_at(key_mid)
    switching_key = key_at(moduli_id)
    b_next = uniform_limbs(rng, moduli[moduli_id + 1:chain], 2, n)
    return dict(key_moduli_id=key_mid, rotation_keys=rotation_keys,
                conjugation_key=conjugation_key, switching_key=switching_key, b_next=b_next)


def codec_values(seed: int, slot_count: int, complex_values: bool) -> np.ndarray:
    """Slot values uniform in [-1, 1) (real and imaginary parts) for codec cases."""
    rng = np.random.default_rng(seed)
    re = rng.uniform(-1.0, 1.0, slot_count)
    if not complex_values:
        return re
    return re + 1j * rng.uniform(-1.0, 1.0, slot_count)


def digest_list(digests) -> str:
    """One digest of an ordered list of digests (a bootstrap stage's diagonals)."""
    return hashlib.sha256("".join(digests).encode()).hexdigest()


def digest_doubles(a) -> str:
    """Digest of the IEEE bit patterns of a float64 / complex128 array."""
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.view(np.uint8).tobytes()).hexdigest()


def arith_inputs(seed: int, moduli, n: int, moduli_id: int, special: int):
    """Operands of the arithmetic cases at `moduli_id` (uniform residues): two
    2-polynomial texts, one a level lower, a 3-polynomial text, a plaintext and a
    relinearization key."""
    rng = np.random.default_rng(seed + 200000)
    chain = len(moduli) - special
    qs = moduli[moduli_id:chain]
    dnum = (chain - moduli_id + special - 1) // special
    return dict(a=uniform_limbs(rng, qs, 2, n), b=uniform_limbs(rng, qs, 2, n),
                low=uniform_limbs(rng, moduli[moduli_id + 1:chain], 2, n),
                trio=uniform_limbs(rng, qs, 3, n), plain=uniform_limbs(rng, qs, 1, n),
                key=uniform_limbs(rng, moduli[moduli_id:], 2 * dnum, n))
