"""Failure paths of the device engine, made to happen without a GPU fault.

The INT8 tensor-core kernels wait on an mbarrier for each MMA round with a bounded
number of polls.  With the limit set to 0 the first wait gives up at once: the
kernel sets the engine's error flag, still drains its MMAs (full limit) before it
frees its tensor memory, and returns.  The host learns of it at the next
synchronize; the context stays usable and, with the limit restored, the same call
gives the right words again."""
import numpy as np
import pytest

from inputs import uniform_limbs

pytestmark = pytest.mark.gpu

NTT, SPECIAL, RELIN = 2, 16, 3


@pytest.mark.parametrize("K", [4, 10])
def test_tensor_core_wait_that_runs_out_is_reported_then_recovers(K):
    from fhe_b200 import Engine, FheError

    e = Engine(log_coeff_count=14 if K == 4 else 16, special_prime_count=K)
    mid = e.moduli_id(e.max_key_switching_level)
    L = e.chains(mid)
    rng = np.random.default_rng(31 + K)
    key = uniform_limbs(rng, e.moduli[mid:], 2 * e.partition_count(mid), e.coeff_count)
    rk = e.upload(key, mid, NTT | SPECIAL, RELIN)
    t3 = uniform_limbs(rng, e.moduli[mid:mid + L], 3, e.coeff_count)
    e.set_tensor_cores(0)
    want = e.relinearize(e.upload(t3, mid, NTT), rk).download()
    e.set_tensor_cores(1)  # both base conversions on the tensor pipe
    assert np.array_equal(e.relinearize(e.upload(t3, mid, NTT), rk).download(), want)

    ct = e.upload(t3, mid, NTT)
    e.synchronize()
    e.set_tensor_core_wait_limit(0)
    with pytest.raises(FheError, match="tensor-core wait ran out"):
        e.relinearize(ct, rk)
        e.synchronize()
    e.synchronize()  # the flag was cleared when it was reported

    e.set_tensor_core_wait_limit(-1)
    for _ in range(2):
        assert np.array_equal(e.relinearize(e.upload(t3, mid, NTT), rk).download(), want)
    e.set_tensor_cores(2)
    e.close()


def test_wait_limit_is_checked():
    from fhe_b200 import Engine, FheError

    e = Engine(log_coeff_count=14, special_prime_count=1)
    with pytest.raises(FheError):
        e.set_tensor_core_wait_limit(1 << 40)
    e.set_tensor_core_wait_limit(-1)
    e.close()
