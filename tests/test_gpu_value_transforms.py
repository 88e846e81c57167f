"""Multiply-then-relinearize with value-only transforms gives the same words as with
the reference's butterflies on every limb.

Relinearization reduces its output to [0, q) and reads most of the product's words
only modulo q; the limbs it reads word for word are each key-switching partition's
first limb of the tensor's third polynomial (Garner's first digit), or all of a
partition's limbs where its first prime exceeds twice another of its primes (the
60-bit first prime of the top level).  With the switch on (the default) the inputs'
rescale-and-transform and the tensor's inverse transform take Harvey's butterflies
on Shoup twiddles on the other limbs, and the tensor's first two polynomials are
folded into the key inner product as P d0, P d1 (ModDown(acc + P d) = ModDown(acc)
+ d) instead of being transformed and added after ModDown; off, every limb is exact
and the addend is added in ModDown's store.  A three-polynomial text being
relinearized has its c0, c1 folded the same way (P c0, P c1).  At the top level of the 10-special-prime
chain the first prime is also a special prime, so P vanishes modulo it and the fold
is not taken there.  The recorded reference digests run with the switch on."""
import numpy as np
import pytest

from inputs import uniform_limbs

pytestmark = pytest.mark.gpu

NTT, RESCALED, SPECIAL = 2, 4, 16
RELIN = 3

CONFIGS = [  # (log_n, special primes, preset, moduli ids)
    (16, 10, 1, [0, 1, 5, 12]),
    (16, 4, 2, [0, 2, 20]),
    (14, 1, 1, [0, 1, 4]),
    (15, 2, 1, [0, 1, 7]),
]


def lazy(rng, limbs, moduli):
    """The same values with about half the words moved to [q, 2q), the engine's
    lazy range."""
    out = limbs.copy()
    for j, q in enumerate(moduli):
        pick = rng.random(out[:, j].shape) < 0.5
        out[:, j][pick] += np.int64(q)
    return out


def both(e, fn):
    e.set_value_transforms(True)
    try:
        fast = fn()
    finally:
        e.set_value_transforms(False)
    try:
        exact = fn()
    finally:
        e.set_value_transforms(True)
    return fast, exact


@pytest.mark.parametrize("log_n,K,preset,mids", CONFIGS, ids=lambda v: str(v))
def test_value_transforms_give_the_same_words(engines, log_n, K, preset, mids):
    e = engines(log_n, K, preset)
    n = e.coeff_count
    for mid in mids:
        rng = np.random.default_rng(7100 + 100 * log_n + 10 * K + mid)
        moduli = e.moduli[mid:e.chain_count]
        a = uniform_limbs(rng, moduli, 2, n)
        b = uniform_limbs(rng, moduli, 2, n)
        key = uniform_limbs(rng, e.moduli[mid:], 2 * e.partition_count(mid), n)
        rk = e.upload(key, mid, NTT | SPECIAL, RELIN)
        la, lb = lazy(rng, a, moduli), lazy(rng, b, moduli)
        t3 = uniform_limbs(rng, moduli, 3, n)
        lt3 = lazy(rng, t3, moduli)

        def ops():
            out = []
            for c in (t3, lt3):
                # A three-polynomial text: its c0, c1 enter the key inner product.
                out.append(e.relinearize(e.upload(c, mid, NTT), rk).download())
                out.append(e.relinearize(e.upload(c, mid), rk).download())
            for x, y in ((a, b), (la, lb)):
                if e.chain_count - mid >= 2:
                    # Rescaled inputs are transformed as they are: the product is at `mid`.
                    out.append(e.multiply(e.upload(x, mid, RESCALED), e.upload(y, mid, RESCALED),
                                          rk).download())
                if e.chain_count - mid >= 3:
                    out.append(e.multiply(e.upload(x, mid), e.upload(y, mid), rk).download())
                    out.append(e.multiply_relinearize_rescale(e.upload(x, mid), e.upload(y, mid),
                                                              rk).download())
                    out.append(e.multiply_relinearize_rescale(e.upload(x, mid, NTT),
                                                              e.upload(y, mid, NTT), rk).download())
            return out

        for tc in (True, False):
            e.set_tensor_cores(tc)
            try:
                fast, exact = both(e, ops)
            finally:
                e.set_tensor_cores(2)
            assert len(fast) == len(exact) > 0
            for i, (got, want) in enumerate(zip(fast, exact)):
                assert np.array_equal(got, want), (mid, tc, i)


@pytest.mark.parametrize("log_n,K,preset,key_mid,mid", [(16, 10, 1, 1, 5), (16, 4, 2, 2, 9)],
                         ids=lambda v: str(v))
def test_value_transforms_with_a_key_above_the_text(engines, log_n, K, preset, key_mid, mid):
    """A relinearization key made at a higher level than the texts: the partitions'
    key rows are offset, the folded addend and the exact limbs are not."""
    e = engines(log_n, K, preset)
    n = e.coeff_count
    rng = np.random.default_rng(7300 + 100 * log_n + 10 * key_mid + mid)
    moduli = e.moduli[mid:e.chain_count]
    a = uniform_limbs(rng, moduli, 2, n)
    b = uniform_limbs(rng, moduli, 2, n)
    t3 = uniform_limbs(rng, moduli, 3, n)
    key = uniform_limbs(rng, e.moduli[key_mid:], 2 * e.partition_count(key_mid), n)
    rk = e.upload(key, key_mid, NTT | SPECIAL, RELIN)

    def ops():
        return [e.multiply_relinearize_rescale(e.upload(a, mid), e.upload(b, mid), rk).download(),
                e.multiply(e.upload(a, mid, RESCALED), e.upload(b, mid, RESCALED), rk).download(),
                e.relinearize(e.upload(t3, mid, NTT), rk).download()]

    fast, exact = both(e, ops)
    for i, (got, want) in enumerate(zip(fast, exact)):
        assert np.array_equal(got, want), i
