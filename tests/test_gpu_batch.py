"""The batched serving step (multiply-relinearize-rescale then a rotation per item, at
uneven levels) gives the words of the same operations called one by one, on its
direct first run, its captured second run and its replays."""
import numpy as np
import pytest

from inputs import uniform_limbs

pytestmark = pytest.mark.gpu

NTT, SPECIAL = 2, 16
RELIN = 3


def test_multiply_rotate_batch_matches_single_operations(engines):
    e = engines(16, 10, 1)
    n = e.coeff_count
    top = e.moduli_id(e.max_key_switching_level)
    rng = np.random.default_rng(4321)
    key = uniform_limbs(rng, e.moduli[top:], 2 * e.partition_count(top), n)
    rk = e.upload(key, top, NTT | SPECIAL, RELIN)
    deltas = [1, 4, 512, 1 << 14]
    rot = {d: e.upload_fixed_rotation_key(
        uniform_limbs(rng, e.moduli[top:], 2 * e.partition_count(top), n), top, d) for d in deltas}
    levels = [24, 2, 13, 7, 24, 19]
    items = []
    for i, level in enumerate(levels):
        mid = e.moduli_id(level)
        q = e.moduli[mid:e.chain_count]
        a = e.upload(uniform_limbs(rng, q, 2, n), mid)
        b = e.upload(uniform_limbs(rng, q, 2, n), mid)
        items.append((a, b, rot[deltas[i % len(deltas)]]))

    want = [e.rotate(e.multiply_relinearize_rescale(a, b, rk), k).download() for a, b, k in items]
    captured_before = e.graph_counts()[0]
    for run in range(3):
        got = e.multiply_rotate_batch([t[0] for t in items], [t[1] for t in items], rk,
                                      [t[2] for t in items])
        assert len(got) == len(items)
        for g, w in zip(got, want):
            assert np.array_equal(g.download(), w), run
    assert e.graph_counts() == (captured_before + 1, 0)


@pytest.mark.parametrize("streams", [1, 3, 8])
def test_multiply_relinearize_rescale_batch_matches_single_operations(engines, streams):
    e = engines(16, 10, 1)
    n = e.coeff_count
    top = e.moduli_id(e.max_key_switching_level)
    rng = np.random.default_rng(99 + streams)
    key = uniform_limbs(rng, e.moduli[top:], 2 * e.partition_count(top), n)
    rk = e.upload(key, top, NTT | SPECIAL, RELIN)
    pairs = []
    for level in [24, 3, 24, 11, 17, 24, 5]:
        mid = e.moduli_id(level)
        q = e.moduli[mid:e.chain_count]
        pairs.append((e.upload(uniform_limbs(rng, q, 2, n), mid),
                      e.upload(uniform_limbs(rng, q, 2, n), mid)))
    want = [e.multiply_relinearize_rescale(a, b, rk).download() for a, b in pairs]
    e.set_concurrency(streams)
    try:
        for run in range(2):
            got = e.multiply_relinearize_rescale_batch([p[0] for p in pairs],
                                                       [p[1] for p in pairs], rk)
            for g, w in zip(got, want):
                assert np.array_equal(g.download(), w), run
    finally:
        e.set_concurrency(4)


def test_concurrency_bounds(engines):
    e = engines(16, 10, 1)
    for bad in (0, 9):
        with pytest.raises(Exception):
            e.set_concurrency(bad)
    e.set_concurrency(4)
