"""A CPU model of the tensor-core NTT (fhe_b200/csrc/ntt_tc.cu), step for step: the
kernel's tile addressing, the byte-split INT8 contraction (exact partial sums per
byte column, folded), the REDC of the fold, the step and pass twists and the staged
stores, checked against the oracle's transforms modulo q at N = 2^16, with every
global address and tile row checked against its bounds.  The GPU suite checks the
kernel itself through every key switch it serves (tests/test_gpu_tensor_core.py)."""
import ctypes

import numpy as np
import pytest

from oracle import oracle

N = 1 << 16
R = 1 << 62
MASK62 = R - 1


def br8(v):
    return int(format(v, "08b")[::-1], 2)


def redc(x, q, k):
    s = ((x & ((1 << 64) - 1)) * k) & MASK62
    z = x + s * q
    assert z % R == 0
    return z >> 62


def tables(q, psi):
    """psi^e R mod q (e < N) and the four matrices M R mod q of make_tc_ntt_tables."""
    r = R % q
    pw, v = [0] * N, r
    for e in range(N):
        pw[e] = v
        v = v * psi % q
    psi_inv = pow(psi, q - 2, q)
    scale = pow(N % q, q - 2, q) * pow(r, q - 2, q) % q
    mats = []
    for mtx in range(4):
        m = [[0] * 16 for _ in range(16)]
        for i in range(16):
            for o in range(16):
                if mtx == 0:
                    val = pow(psi, 4096 * (2 * o + 1) * i, q)
                elif mtx == 1:
                    val = pow(psi, 8192 * i * o, q)
                elif mtx == 2:
                    val = pow(psi_inv, 8192 * i * o, q)
                else:
                    val = pow(psi_inv, 4096 * o * (2 * i + 1), q) * scale % q
                m[i][o] = val * r % q
        mats.append(m)
    return pw, mats


def psi_power(pw, e, q):
    e &= 2 * N - 1
    if e < N:
        return pw[e]
    t = pw[e - N]
    return 0 if t == 0 else q - t


def contract(vals, m, q):
    """The fold of the 8 byte-column partial sums: sum_in sum_byte v[byte] (M 2^(8 byte))."""
    outs = []
    for o in range(16):
        x = 0
        for i in range(16):
            e = m[i][o]
            for byte in range(8):
                part = ((vals[i] >> (8 * byte)) & 255) * e
                x += part
                e = (e << 8) % q
        assert x < 1 << 80
        outs.append(x)
    return outs


def run_pass(kind, x, q, k, pw, mats):
    ma = {0: 0, 1: 1, 2: 2, 3: 2}[kind]
    mb = {0: 1, 1: 1, 2: 2, 3: 3}[kind]
    for blk in range(32):
        line0 = blk * 8
        a_rows = [[None] * 16 for _ in range(128)]
        for idx in range(2048):  # tile_input
            if kind == 0:
                line, m = idx & 7, idx >> 3
                addr = m * 256 + line0 + line
            elif kind == 3:
                line, pb = idx & 7, idx >> 3
                m = br8(pb)
                addr = pb * 256 + line0 + line
            else:
                line, j = idx >> 8, idx & 255
                m = br8(j) if kind == 2 else j
                addr = (line0 + line) * 256 + j
            assert 0 <= addr < N
            row = (m & 15) * 8 + line
            assert a_rows[row][m >> 4] is None
            a_rows[row][m >> 4] = x[addr] % q if x[addr] < 0 else x[addr]
        a2_rows = [[None] * 16 for _ in range(128)]
        for row in range(128):
            a, line = row >> 3, row & 7
            xs = contract(a_rows[row], mats[ma], q)
            for c in range(16):
                u = redc(xs[c], q, k)
                assert u < q + (1 << 18)
                e = [256 * (2 * c + 1) * a, 512 * c * a, -512 * c * a, -256 * (2 * a + 1) * c][kind]
                assert a2_rows[c * 8 + line][a] is None
                a2_rows[c * 8 + line][a] = redc(u * psi_power(pw, e, q), q, k)
        stage = [None] * 2048
        for row in range(128):
            c, line = row >> 3, row & 7
            big_l = line0 + line
            xs = contract(a2_rows[row], mats[mb], q)
            for d in range(16):
                o = c + 16 * d
                w = redc(xs[d], q, k)
                if kind == 0:
                    w = redc(w * psi_power(pw, (2 * o + 1) * big_l, q), q, k)
                    s = br8(o) * 8 + line
                elif kind == 1:
                    s = line * 256 + br8(o)
                elif kind == 2:
                    w = redc(w * psi_power(pw, -(2 * br8(big_l) + 1) * o, q), q, k)
                    s = line * 256 + o
                else:
                    w = w - q if w >= q else w
                    s = o * 8 + line
                assert stage[s] is None
                stage[s] = w
        for idx in range(2048):
            if kind in (0, 3):
                addr = (idx >> 3) * 256 + line0 + (idx & 7)
            else:
                addr = (line0 + (idx >> 8)) * 256 + (idx & 255)
            assert 0 <= addr < N
            x[addr] = stage[idx]


@pytest.fixture(scope="module")
def prime():
    from fhe_b200 import _lib

    cfg = _lib.FheConfig(16, -1, 10, -1, 1)
    info = _lib.FheEngineInfo()
    qbuf = (ctypes.c_uint64 * 64)()
    _lib.check(_lib.load().fhe_parameters_query(ctypes.byref(cfg), ctypes.byref(info), qbuf, 64))
    qs = np.array(qbuf[: info.prime_count], dtype=np.uint64)
    ctx = oracle.Context(16, qs, 10)
    t = ctx.tables()
    i = 3
    q, k = int(qs[i]), int(t["k"][i])
    root, root_inverse = t["root"][i], t["root_inverse"][i]
    e1 = np.zeros(N, dtype=np.int64)
    e1[1] = 1
    psi = int(oracle.ntt_limb(e1, root, q, k)[0]) % q  # position 0 holds psi^1
    return q, k, root, root_inverse, psi


def test_forward_model_matches_the_reference_transform_mod_q(prime):
    q, k, root, _, psi = prime
    pw, mats = tables(q, psi)
    x0 = np.random.default_rng(7).integers(0, 2 * q, size=N, dtype=np.int64)
    want = oracle.ntt_limb(x0.copy(), root, q, k).astype(object) % q
    x = [int(v) for v in x0]
    run_pass(0, x, q, k, pw, mats)
    run_pass(1, x, q, k, pw, mats)
    assert all(v < 2 * q for v in x)
    assert all(x[p] % q == int(want[p]) for p in range(N))


def test_inverse_model_matches_the_reference_enter_exit_transform(prime):
    q, k, _, root_inverse, psi = prime
    pw, mats = tables(q, psi)
    xh = np.random.default_rng(8).integers(0, q, size=N, dtype=np.int64)
    want = oracle.intt_limb(xh.copy(), root_inverse, q, k).astype(object) % q
    scale = pow(N, q - 2, q) * pow(R % q, q - 2, q) % q  # to_intt_'s enter-exit
    y = [int(v) for v in xh]
    run_pass(2, y, q, k, pw, mats)
    run_pass(3, y, q, k, pw, mats)
    assert all(y[i] == int(want[i]) * scale % q for i in range(N))
