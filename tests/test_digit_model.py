"""Which words of a relinearized polynomial Garner's digits read exactly, checked on the
CPU against the oracle's restatement of the reference's rns_to_mrs
(core_key_switch.cpp:21-56).

The engine transforms a product value-only except each key-switching partition's
first limb (ExactLimbs): the first digit is that limb's word itself, while limb j > 0
enters as guard(x_j + 2q_j - Y, 2q_j), a Montgomery product and a reduction to
[0, q_j), whose result depends on x_j only modulo q_j while 0 <= Y <= 2q_j, which
holds when the partition's first prime is at most twice each of its others.  So:
moving words of the other limbs from x to x + q leaves every digit unchanged in such
a partition, while moving first-limb words changes them; a partition whose first
prime is larger (the 60-bit first prime at the top level) is kept exact whole."""
import numpy as np
import pytest

from inputs import TIERS, uniform_limbs
from oracle import oracle
from test_params import query

CASES = [("silver", [0, 1, 5]), ("gold", [0, 1, 9]), ("c10", [0, 1, 12]),
         ("bootstrap_gold", [0, 2, 20])]


def partitions(L: int, K: int):
    """(start, size) of each partition at L limbs (ckks/parameters.cpp:334-360)."""
    pc = (L + K - 1) // K
    return [(max(0, s), min(L, s + K) - max(0, s)) for s in range(L - pc * K, L, K)]


def lazy_words(rng, x, limbs, moduli):
    """x with about half the words of the given limbs moved to [q, 2q)."""
    y = x.copy()
    for j in limbs:
        pick = rng.random(x.shape[1]) < 0.5
        y[j][pick] += np.int64(moduli[j])
    return y


@pytest.mark.parametrize("tier,mids", CASES, ids=[c[0] for c in CASES])
def test_digits_read_first_limbs_exactly_and_others_by_value(tier, mids):
    log_n, K, preset = TIERS[tier]
    info, q = query(log_n, K, preset)
    q = [int(v) for v in q]
    chain = len(q) - K
    ctx = oracle.Context(log_n, q, K)
    n = 1 << log_n
    for mid in mids:
        rng = np.random.default_rng(5500 + 100 * log_n + 10 * K + mid)
        L = chain - mid
        moduli = q[mid:chain]
        x = uniform_limbs(rng, moduli, 1, n)[0]
        want = ctx.mixed_radix(mid, mid, x)
        parts = partitions(L, K)
        bounded = [all(moduli[s] <= 2 * moduli[s + j] for j in range(1, size)) for s, size in parts]

        others = [s + j for s, size in parts for j in range(1, size)]
        got = ctx.mixed_radix(mid, mid, lazy_words(rng, x, others, moduli))
        for (s, size), ok in zip(parts, bounded):
            if ok:
                assert np.array_equal(got[s:s + size], want[s:s + size]), (tier, mid, s)

        firsts = [s for s, size in parts if size > 1]
        if firsts:
            moved = ctx.mixed_radix(mid, mid, lazy_words(rng, x, firsts, moduli))
            assert not np.array_equal(moved, want), (tier, mid)
