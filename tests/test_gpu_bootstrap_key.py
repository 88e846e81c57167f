"""GPU parity of bootstrapping with a bootstrap key (the hoisted baby-step giant-step
form): the bootstrap preset at N = 2^16 with 4 special primes, a "medium" key of 3
stages made on the device from the reseeded random stream.  Every fixed rotation
key, every stage's diagonals, the small bootstrap key and the bootstrapped
ciphertext must equal the reference's words; the decoded slots keep its precision."""
import numpy as np
import pytest

from conftest import load_golden
from inputs import codec_values, digest, digest_doubles, digest_list

pytestmark = pytest.mark.gpu

CASES = load_golden("bootstrap_key.json")


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["tier"])
def test_bootstrap_key_matches_recorded_reference(engines, case):
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

    bk = e.create_bootstrap_key(sk, case["stage_count"], case["size"])
    info = bk.info()
    assert info["stage_count"] == case["stage_count"]
    assert info["rotation_key_count"] == len(case["rotation_keys"])
    assert bk.deltas() == [delta for delta, _ in case["rotation_keys"]]
    for delta, want in case["rotation_keys"]:
        assert digest(bk.rotation_key(delta).download()) == want, delta
    for st in case["stages"]:
        level, inner, outer = bk.stage(bool(st["to_slot"]), st["stage"])
        assert (level, inner, outer) == (st["level"], st["inner"], st["outer"])
        digests = []
        for o in range(outer):
            for i in range(inner):
                diag = bk.diagonal(bool(st["to_slot"]), st["stage"], o, i)
                if diag is not None:
                    digests.append(digest(diag.download()))
        assert len(digests) == st["diagonal_count"]
        assert digest_list(digests) == st["diagonals"], (st["to_slot"], st["stage"])
    to_sparse, to_dense = bk.small_bootstrap_key()
    assert digest(to_sparse.download()) == d["to_sparse"]
    assert digest(to_dense.download()) == d["to_dense"]

    vals = codec_values(case["values_seed"], e.slot_count, True)
    ct = e.encrypt(e.encode(vals, case["encrypt_level"]), sk)
    assert digest(ct.download()) == d["ciphertext"]
    out = e.bootstrap(ct, rk, ck, bk)
    info = out.info()
    assert (info["moduli_id"], info["level"]) == (case["output_moduli_id"], case["output_level"])
    assert digest(out.download()) == d["bootstrapped"]
    slots = e.decode(e.decrypt(out, sk), complex_output=True)
    assert digest_doubles(slots) == case["decoded"]
    assert np.max(np.abs(slots - vals)) < 2.0 ** -16

    # The second call captures the bootstrap as a CUDA graph, the third replays it;
    # with graphs off the direct path runs again.  Same words every time.
    before = e.kernel_launch_count()
    for _ in range(2):
        again = e.bootstrap(ct, rk, ck, bk)
        assert digest(again.download()) == d["bootstrapped"]
    assert e.kernel_launch_count() > before
    assert e.graph_counts() == (1, 0)
    e.set_graphs(False)
    try:
        assert digest(e.bootstrap(ct, rk, ck, bk).download()) == d["bootstrapped"]
        # The linear transforms' inner loops as per-rotation kernels instead of the
        # fused kernel: the same words.
        e.set_fused_bsgs(False)
        assert digest(e.bootstrap(ct, rk, ck, bk).download()) == d["bootstrapped"]
    finally:
        e.set_fused_bsgs(True)
        e.set_graphs(True)

    # A batch runs its bootstraps on several streams (each stream with graphs of its
    # own after its first direct run): the words of the single calls.
    ct2 = e.encrypt(e.encode(codec_values(case["values_seed"] + 1, e.slot_count, True),
                             case["encrypt_level"]), sk)
    want2 = digest(e.bootstrap(ct2, rk, ck, bk).download())
    batch = [ct, ct2, ct]
    for run in range(3):
        got = [digest(o.download()) for o in e.bootstrap_batch(batch, rk, ck, bk)]
        assert got == [d["bootstrapped"], want2, d["bootstrapped"]], run


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["tier"])
def test_bootstrap_key_rejects_bad_arguments(engines, case):
    from fhe_b200._lib import FheError

    e = engines(case["log_n"], case["special_prime_count"], case["preset"])
    sk = e.create_secret_key()
    with pytest.raises(FheError, match="Create Bootstrap Key: invalid size."):
        e.create_bootstrap_key(sk, 3, "huge")
    with pytest.raises(FheError, match="Create Bootstrap Key: invalid stage count."):
        e.create_bootstrap_key(sk, 2, "medium")
