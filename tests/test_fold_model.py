"""The identity behind folding a product's first two polynomials (or a relinearized
text's c0, c1) into the key inner product, checked on the CPU against the oracle's
restatement of the reference's ModDown (core_key_switch.cpp:110-160) and of
relinearize's addition after it (core.cpp:713-741):

    reduce(to_intt(d) + mod_down(acc)) == mod_down(acc + P d)

word for word, where acc is an NTT-form accumulator over every prime of the level, d
an NTT-form addend on its normal limbs (words in [0, 2q), as the engine's transforms
leave them) and P the product of the special primes.  The engine adds P d inside the
key inner product's exact sums; the identity also shows where it must not: a level
whose normal primes include a special prime (the top level of the 10-special-prime
chain), where P is 0 modulo that prime and d would be lost."""
import numpy as np
import pytest

from inputs import TIERS, uniform_limbs
from oracle import oracle
from test_params import query

CASES = [("bronze", [0, 3]), ("silver", [0, 5]), ("gold", [0, 9]), ("c10", [0, 1, 12])]


def mulmod_rows(x: np.ndarray, c: list, moduli: list) -> np.ndarray:
    """(x[j] * c[j]) mod moduli[j] per limb, exactly (Python integers)."""
    out = np.empty_like(x)
    for j, (cj, q) in enumerate(zip(c, moduli)):
        out[j] = np.array([(int(v) * cj) % q for v in x[j].tolist()], dtype=np.int64)
    return out


@pytest.mark.parametrize("tier,mids", CASES, ids=[c[0] for c in CASES])
def test_mod_down_of_folded_addend_matches_addition_after_mod_down(tier, mids):
    log_n, K, preset = TIERS[tier]
    info, q = query(log_n, K, preset)
    q = [int(v) for v in q]
    chain = len(q) - K
    specials = q[chain:]
    P = 1
    for p in specials:
        P *= p
    ctx = oracle.Context(log_n, q, K)
    n = 1 << log_n
    for mid in mids:
        rng = np.random.default_rng(4400 + 100 * log_n + 10 * K + mid)
        L = chain - mid
        normal = q[mid:chain]
        acc = uniform_limbs(rng, q[mid:], 1, n)[0]
        d = uniform_limbs(rng, normal, 1, n)[0]
        d = d + np.where(rng.random(d.shape) < 0.5, np.array(normal, dtype=np.int64)[:, None], 0)

        # The reference: transform d back and add it after ModDown, reduced to [0, q).
        want = ctx.to_intt(mid, d[None])[0] + ctx.mod_down(mid, acc)
        qs = np.array(normal, dtype=np.int64)[:, None]
        want = np.where(want >= 2 * qs, want - 2 * qs, want)
        want = np.where(want >= qs, want - qs, want)

        # The fold: P d added to the accumulator's normal limbs before ModDown.
        folded = acc.copy()
        folded[:L] = (mulmod_rows(d, [P % p for p in normal], normal) + acc[:L]) % qs
        got = ctx.mod_down(mid, folded)

        if any(p in specials for p in normal):
            # P vanishes modulo the special prime in the chain: the addend is lost there.
            lost = [j for j, p in enumerate(normal) if p in specials]
            assert not np.array_equal(got[lost], want[lost])
            keep = [j for j in range(L) if j not in lost]
            assert np.array_equal(got[keep], want[keep])
        else:
            assert np.array_equal(got, want), (tier, mid)
