"""The product's host parameter layer (C++, reached through the C ABI's host-only
queries) against the reference's known answers and the oracle."""
import ctypes

import numpy as np
import pytest

from conftest import load_golden
from inputs import TIERS
from fhe_b200 import _lib
from oracle import oracle


def query(log_n, K, preset, max_level=-1, log_slot=-1):
    lib = _lib.load()
    cfg = _lib.FheConfig(log_n, log_slot, K, max_level, preset)
    info = _lib.FheEngineInfo()
    q = (ctypes.c_uint64 * 256)()
    _lib.check(lib.fhe_parameters_query(ctypes.byref(cfg), ctypes.byref(info), q, 256))
    return info, np.array(q[: info.prime_count], dtype=np.uint64)


def tables(log_n, K, preset):
    lib = _lib.load()
    info, q = query(log_n, K, preset)
    P, n = info.prime_count, 1 << log_n
    k = np.empty(P, dtype=np.uint64)
    r2 = np.empty(P, dtype=np.int64)
    ni = np.empty(P, dtype=np.int64)
    root = np.empty((P, n - 1), dtype=np.int64)
    rinv = np.empty((P, n - 1), dtype=np.int64)
    ip = _lib._i64p
    cfg = _lib.FheConfig(log_n, -1, K, -1, preset)
    _lib.check(lib.fhe_parameters_tables(ctypes.byref(cfg), k.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                         r2.ctypes.data_as(ip), ni.ctypes.data_as(ip),
                                         root.ctypes.data_as(ip), rinv.ctypes.data_as(ip)))
    return dict(q=q, k=k, r_squared=r2, n_inverse=ni, root=root, root_inverse=rinv)


KATS = load_golden("precomputed_kat.json")


@pytest.mark.parametrize("name", sorted(KATS))
def test_chain_and_tables_match_precomputed_known_answers(name):
    entry = KATS[name]
    log_n, K, preset = TIERS[entry["tier"]]
    v = entry["vectors"]
    t = tables(log_n, K, preset)
    # the reference's vectors are the full chain (q) or a prefix of each table
    assert t["q"].tolist() == v["q"]

    def prefix(a, name):
        return a.reshape(-1)[: len(v[name])].tolist()

    assert prefix(t["q"] * 2, "q_double") == v["q_double"]
    assert prefix(t["q"] >> 1, "q_half") == v["q_half"]
    assert prefix(t["k"], "k") == v["k"]
    assert prefix(t["r_squared"], "r_squared") == v["r_squared"]
    assert prefix(t["n_inverse"], "coeff_count_inverse") == v["coeff_count_inverse"]
    assert t["root"].reshape(-1)[: len(v["root"])].tolist() == v["root"]
    assert t["root_inverse"].reshape(-1)[: len(v["root_inverse"])].tolist() == v["root_inverse"]


@pytest.mark.parametrize("tier", ["sand", "pebble", "iron", "bronze"])
def test_tables_match_oracle(tier):
    log_n, K, preset = TIERS[tier]
    t = tables(log_n, K, preset)
    o = oracle.Context(log_n, t["q"], K).tables()
    for key in ("k", "r_squared", "n_inverse", "root", "root_inverse"):
        assert np.array_equal(t[key], o[key]), key


def test_config_c_key_switching_shape():
    """N=2^16 with 10 special primes: 29-limb chain, key switching at 28 limbs, dnum 3."""
    info, q = query(16, 10, 1)
    assert (info.chain_count, info.prime_count, info.full_level) == (29, 39, 27)
    assert info.max_key_switching_level == 26
    assert all(int(p) % (2 << 16) == 1 for p in q)
    # the one-more-level prime repeats the first special prime
    assert q[0] == q[info.chain_count]


@pytest.mark.parametrize("log_n,K,preset,msg", [
    (12, 1, 1, "log coefficient count is too small"),
    (18, 1, 1, "log coefficient count is too large"),
    (15, 1, 2, "log coefficient count is too small"),
    (14, 17, 1, "special prime count is too large"),
    (14, -1, 1, "special prime count is too small"),
])
def test_config_validation_messages(log_n, K, preset, msg):
    with pytest.raises(_lib.FheError) as exc:
        query(log_n, K, preset)
    assert msg in str(exc.value)
    assert exc.value.status == -1


def test_slot_count_and_max_level():
    info, _ = query(14, 1, 1, max_level=3, log_slot=10)
    assert info.slot_count == 1024
    assert info.max_level == 3
    assert info.max_key_switching_level == 3
