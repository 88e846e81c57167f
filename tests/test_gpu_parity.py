"""GPU parity: the sm_100a kernels, called through the C ABI, against the recorded
reference outputs and the CPU oracle.  Integer work must be bit-exact."""
import numpy as np
import pytest

from conftest import load_golden
from inputs import TIERS, case_inputs, digest, uniform_limbs
from oracle import oracle

pytestmark = pytest.mark.gpu

NTT, RESCALED, SPECIAL = 2, 4, 16


CASES = load_golden("ref_ops.json")


HEADLINE_CASES = load_golden("ref_ops_c10.json")


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c['tier']}-m{c['moduli_id']}")
def test_ops_match_recorded_reference(engines, case):
    check_core_ops(engines(case["log_n"], case["special_prime_count"], case["preset"]), case)


@pytest.mark.parametrize("mode", [1, 0], ids=["tensor-cores", "cuda-cores"])
@pytest.mark.parametrize("case", HEADLINE_CASES, ids=lambda c: f"{c['tier']}-m{c['moduli_id']}")
def test_headline_ops_match_recorded_reference(engines, case, mode):
    """N = 2^16 with 10 special primes (dnum = 3, up to 10-limb partitions), against
    the reference's own words, with both base conversions forced onto the INT8
    tensor pipe and then onto the CUDA cores."""
    e = engines(case["log_n"], case["special_prime_count"], case["preset"])
    e.set_tensor_cores(mode)
    try:
        check_core_ops(e, case)
    finally:
        e.set_tensor_cores(2)


def check_core_ops(e, case):
    from fhe_b200 import RELINEARIZATION_KEY

    q = np.array(case["moduli"], dtype=np.uint64)
    assert e.moduli.tolist() == case["moduli"]
    mid = case["moduli_id"]
    K = case["special_prime_count"]
    a, b, ct3, key = case_inputs(case["seed"], q, e.coeff_count, mid, K)
    rk = e.upload(key, mid, NTT | SPECIAL, RELINEARIZATION_KEY)
    d = case["digests"]

    assert digest(e.ntt(e.upload(a, mid)).download()) == d["to_ntt"]
    assert digest(e.intt(e.upload(a, mid, NTT)).download()) == d["to_intt"]
    assert digest(e.relinearize(e.upload(ct3, mid, NTT), rk).download()) == d["relinearize"]
    if e.chains(mid) >= 3:
        assert digest(e.rescale(e.upload(a, mid)).download()) == d["rescale"]
    if e.chains(mid) >= 2:
        t = e.multiply(e.upload(a, mid, NTT | RESCALED), e.upload(b, mid, NTT | RESCALED))
        assert digest(t.download()) == d["tensor"]
    if "mult_relin_rescale" in d:
        fused = e.multiply_relinearize_rescale(e.upload(a, mid), e.upload(b, mid), rk)
        assert digest(fused.download()) == d["mult_relin_rescale"]
        stepwise = e.rescale(e.multiply(e.upload(a, mid), e.upload(b, mid), rk))
        assert digest(stepwise.download()) == d["mult_relin_rescale"]
        info = fused.info()
        assert info["flag"] & RESCALED and not info["flag"] & NTT


@pytest.fixture(scope="module")
def config_c(engines):
    """N=2^16, 10 special primes: fresh ciphertexts at the key-switching level (28 limbs)."""
    e = engines(16, 10, 1)
    ctx = oracle.Context(16, e.moduli, 10)
    return e, ctx


def test_full_size_mult_relin_rescale_matches_oracle(config_c):
    from fhe_b200 import RELINEARIZATION_KEY

    e, ctx = config_c
    mid = e.moduli_id(e.max_key_switching_level)
    assert e.chains(mid) == 28 and e.partition_count(mid) == 3
    a, b, ct3, key = case_inputs(4242, e.moduli, e.coeff_count, mid, 10)
    rk = e.upload(key, mid, NTT | SPECIAL, RELINEARIZATION_KEY)
    got = e.multiply_relinearize_rescale(e.upload(a, mid), e.upload(b, mid), rk).download()
    want = ctx.mult_relin_rescale(mid, a, b, mid, key)
    assert got.shape == (2, 26, 1 << 16)
    assert np.array_equal(got, want)


def test_full_size_relinearize_matches_oracle(config_c):
    from fhe_b200 import RELINEARIZATION_KEY

    e, ctx = config_c
    mid = 2  # 27 limbs: partitions [7, 10, 10] against a key made at moduli id 1
    key_mid = 1
    rng = np.random.default_rng(99)
    ct3 = uniform_limbs(rng, e.moduli[mid:e.chain_count], 3, e.coeff_count)
    key = uniform_limbs(rng, e.moduli[key_mid:], 2 * e.partition_count(key_mid), e.coeff_count)
    rk = e.upload(key, key_mid, NTT | SPECIAL, RELINEARIZATION_KEY)
    got = e.relinearize(e.upload(ct3, mid, NTT), rk).download()
    assert np.array_equal(got, ctx.relinearize(mid, ct3, key_mid, key))


@pytest.mark.parametrize("batch", [1, 3])
def test_ntt_microbench_shape_matches_oracle(engines, batch):
    """N=2^16, the first 24 primes of the Gold chain, plain per-limb transforms."""
    from fhe_b200 import UNIT_PLAINTEXT

    e = engines(16, 4, 1)
    q = e.moduli[:24]
    rng = np.random.default_rng(7 + batch)
    x = uniform_limbs(rng, q, batch, e.coeff_count)
    tables = oracle.Context(16, e.moduli, 4).tables()
    buf = e.upload(x, e.chain_count - 24, kind=UNIT_PLAINTEXT)  # any 24-limb buffer
    ptr = buf.device_pointer()
    e.ntt_limbs(ptr, 0, 24, batch, 24 << 16, inverse=False)
    got = buf.download()
    for p in range(batch):
        for j in (0, 11, 23):
            want = oracle.ntt_limb(x[p, j], tables["root"][j], int(q[j]), int(tables["k"][j]))
            assert np.array_equal(got[p, j], want), (p, j)
    e.ntt_limbs(ptr, 0, 24, batch, 24 << 16, inverse=True)
    back = buf.download()
    for p in range(batch):
        for j in (0, 23):
            want = oracle.intt_limb(got[p, j], tables["root_inverse"][j], int(q[j]), int(tables["k"][j]))
            assert np.array_equal(back[p, j], want), (p, j)


@pytest.mark.parametrize("log_n", [13, 14, 15, 16, 17])
def test_ntt_round_trip_every_ring_degree(engines, log_n):
    """to_intt(to_ntt(x)) == x (mod q) on every supported ring degree."""
    K = {13: 1, 14: 1, 15: 2, 16: 4, 17: 6}[log_n]
    e = engines(log_n, K, 1)
    mid = e.chain_count - 4
    rng = np.random.default_rng(log_n)
    x = uniform_limbs(rng, e.moduli[mid:e.chain_count], 2, e.coeff_count)
    back = e.intt(e.ntt(e.upload(x, mid))).download()
    q = e.moduli[mid:e.chain_count].astype(np.int64)[None, :, None]
    assert np.array_equal(back % q, x)
    ctx = oracle.Context(log_n, e.moduli, K)
    fwd = e.ntt(e.upload(x, mid)).download()
    assert np.array_equal(fwd, ctx.to_ntt(mid, x))


def test_errors_mirror_reference_messages(engines):
    from fhe_b200 import FheError, RELINEARIZATION_KEY

    e = engines(*TIERS["pebble"])
    mid = e.chain_count - 1  # a single limb: level -1 when not rescaled
    x = uniform_limbs(np.random.default_rng(1), e.moduli[mid:e.chain_count], 2, e.coeff_count)
    with pytest.raises(FheError, match="should have a positive level"):
        e.rescale(e.upload(x, mid))
    y = uniform_limbs(np.random.default_rng(2), e.moduli[3:e.chain_count], 2, e.coeff_count)
    with pytest.raises(FheError, match="should have 3 polynomials"):
        key = uniform_limbs(np.random.default_rng(3), e.moduli[3:], 2 * e.partition_count(3), e.coeff_count)
        e.relinearize(e.upload(y, 3, NTT), e.upload(key, 3, NTT | SPECIAL, RELINEARIZATION_KEY))


def test_mont_mult_limbs_matches_redc(engines):
    """SingleProcessor::mont_mult on device limbs (unit.h:15-23): y = (a b + s q) / 2^62
    with s = (a b mod 2^64) k mod 2^62, k = -q^-1 mod 2^62, in [0, 2q)."""
    import torch

    e = engines(14, 1, 1)
    n, chains, polys = e.coeff_count, 5, 2
    mid = 1
    rng = np.random.default_rng(77)
    qs = [int(q) for q in e.moduli[mid:mid + chains]]
    a = np.stack([np.stack([rng.integers(0, 2 * q, size=n, dtype=np.int64) for q in qs])
                  for _ in range(polys)])
    b = np.stack([np.stack([rng.integers(0, 2 * q, size=n, dtype=np.int64) for q in qs])
                  for _ in range(polys)])
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(b).cuda()
    dy = torch.empty_like(da)
    e.synchronize()
    torch.cuda.synchronize()
    e.mont_mult_limbs(da.data_ptr(), db.data_ptr(), dy.data_ptr(), mid, chains, polys, chains * n)
    e.synchronize()
    got = dy.cpu().numpy()
    R = 1 << 62
    for j, q in enumerate(qs):
        k = (-pow(q, -1, R)) % R
        for p in range(polys):
            for c in range(0, n, 97):
                x = int(a[p, j, c]) * int(b[p, j, c])
                s = ((x % (1 << 64)) * k) % R
                assert int(got[p, j, c]) == (x + s * q) >> 62
