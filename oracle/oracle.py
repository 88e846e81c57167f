"""ctypes bindings for the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the benchmark's CPU-baseline leg may
import this module; it is the checker, never the product path.  Arrays are numpy
int64 in the [poly][limb][N] layout described in ckks_oracle.h.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

_i64p = ctypes.POINTER(ctypes.c_int64)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_lib = None


def build() -> None:
    """Compile liboracle.so with the committed Makefile (gcc only)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        L = _lib
        L.oracle_mont_mult.restype = ctypes.c_int64
        L.oracle_mont_mult.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_uint64, ctypes.c_uint64]
        L.oracle_mont_exit.restype = ctypes.c_int64
        L.oracle_mont_exit.argtypes = [ctypes.c_int64, ctypes.c_uint64, ctypes.c_uint64]
        L.oracle_calculate_k.restype = ctypes.c_uint64
        L.oracle_calculate_k.argtypes = [ctypes.c_uint64]
        L.oracle_find_root.restype = ctypes.c_int64
        L.oracle_find_root.argtypes = [ctypes.c_int64, ctypes.c_int]
        for name in ("oracle_ntt_limb", "oracle_intt_limb"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [_i64p, _i64p, _i64p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        L.oracle_ctx_new.restype = ctypes.c_void_p
        L.oracle_ctx_new.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _u64p]
        L.oracle_ctx_free.restype = None
        L.oracle_ctx_free.argtypes = [ctypes.c_void_p]
        L.oracle_ctx_tables.restype = None
        L.oracle_ctx_tables.argtypes = [ctypes.c_void_p, _u64p, _i64p, _i64p, _i64p, _i64p]
        L.oracle_chain_count.restype = ctypes.c_int
        L.oracle_chain_count.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_partition_count.restype = ctypes.c_int
        L.oracle_partition_count.argtypes = [ctypes.c_void_p, ctypes.c_int]
        for name in ("oracle_to_ntt", "oracle_to_intt"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64p, _i64p]
        L.oracle_tensor.restype = None
        L.oracle_tensor.argtypes = [ctypes.c_void_p, ctypes.c_int, _i64p, _i64p, _i64p]
        L.oracle_relinearize.restype = None
        L.oracle_relinearize.argtypes = [ctypes.c_void_p, ctypes.c_int, _i64p, ctypes.c_int, _i64p, _i64p]
        L.oracle_key_switch.restype = None
        L.oracle_key_switch.argtypes = [ctypes.c_void_p, ctypes.c_int, _i64p, ctypes.c_int, _i64p, _i64p]
        L.oracle_mod_down.restype = None
        L.oracle_mod_down.argtypes = [ctypes.c_void_p, ctypes.c_int, _i64p, _i64p]
        L.oracle_mixed_radix.restype = None
        L.oracle_mixed_radix.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _i64p, _i64p]
        L.oracle_rescale.restype = None
        L.oracle_rescale.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _i64p, _i64p]
        L.oracle_mult_relin_rescale.restype = None
        L.oracle_mult_relin_rescale.argtypes = [ctypes.c_void_p, ctypes.c_int, _i64p, _i64p,
                                                ctypes.c_int, _i64p, _i64p]
        for name in ("oracle_switch_key", "oracle_conjugate"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [ctypes.c_void_p, ctypes.c_int, _i64p, ctypes.c_int, _i64p, _i64p]
        L.oracle_rotate.restype = None
        L.oracle_rotate.argtypes = [ctypes.c_void_p, ctypes.c_int, _i64p, ctypes.c_int, _i64p,
                                    ctypes.c_int, _i64p]
        L.oracle_permutation_and_sign.restype = None
        L.oracle_permutation_and_sign.argtypes = [_i32p, _i32p, ctypes.c_int, ctypes.c_int]
        L.oracle_ntt_permutation.restype = None
        L.oracle_ntt_permutation.argtypes = [_i32p, ctypes.c_int, ctypes.c_int]
        L.oracle_deviations.restype = None
        L.oracle_deviations.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_double)]
        L.oracle_level_down_multiplier.restype = ctypes.c_int
        L.oracle_level_down_multiplier.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64p]
        L.oracle_level_down.restype = None
        L.oracle_level_down.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, _i64p, _i64p, _i64p]
        _f64 = ctypes.POINTER(ctypes.c_double)
        L.oracle_encode_level.restype = None
        L.oracle_encode_level.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_void_p, _f64, _i32p, _i32p, _i64p]
        L.oracle_encode.restype = None
        L.oracle_encode.argtypes = [ctypes.c_void_p, _f64, _f64, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_int, ctypes.c_int, _i64p, ctypes.c_int, _i64p]
        L.oracle_decode_plaintext.restype = None
        L.oracle_decode_plaintext.argtypes = [ctypes.c_void_p, _i64p, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_void_p, ctypes.c_double, _f64, _f64]
        _u32p = ctypes.POINTER(ctypes.c_uint32)
        L.oracle_chacha_block.restype = None
        L.oracle_chacha_block.argtypes = [_u32p, _u32p, ctypes.c_uint64, _u32p]
        L.oracle_rand_int.restype = None
        L.oracle_rand_int.argtypes = [_u32p, _u32p, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64,
                                      ctypes.c_int64, _i64p]
        L.oracle_discrete_gaussian.restype = None
        L.oracle_discrete_gaussian.argtypes = [_u32p, _u32p, ctypes.c_uint64, ctypes.c_int, _u64p,
                                               ctypes.c_int, ctypes.c_int, _i64p]
        for name in ("oracle_rotate_plain", "oracle_rotate_plain_ntt"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64p, _i64p]
    return _lib


def _p(a: np.ndarray, t=_i64p):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(t)


def mont_mult(a: int, b: int, q: int, k: int) -> int:
    return lib().oracle_mont_mult(a, b, q, k)


def mont_exit(a: int, q: int, k: int) -> int:
    return lib().oracle_mont_exit(a, q, k)


def calculate_k(q: int) -> int:
    return lib().oracle_calculate_k(q)


def find_root(q: int, n: int) -> int:
    return lib().oracle_find_root(q, n)


def ntt_limb(x, root, q, k):
    x = np.ascontiguousarray(x, dtype=np.int64)
    root = np.ascontiguousarray(root, dtype=np.int64)
    y = np.empty_like(x)
    n = x.shape[0]
    lib().oracle_ntt_limb(_p(x), _p(y), _p(root), q, k, n, n.bit_length() - 1)
    return y


def intt_limb(x, root_inverse, q, k):
    x = np.ascontiguousarray(x, dtype=np.int64)
    root_inverse = np.ascontiguousarray(root_inverse, dtype=np.int64)
    y = np.empty_like(x)
    n = x.shape[0]
    lib().oracle_intt_limb(_p(x), _p(y), _p(root_inverse), q, k, n, n.bit_length() - 1)
    return y


def permutation_and_sign(n: int, delta: int):
    perm = np.empty(n, dtype=np.int32)
    sign = np.empty(n, dtype=np.int32)
    lib().oracle_permutation_and_sign(_p(perm, _i32p), _p(sign, _i32p), n, delta)
    return perm, sign


def ntt_permutation(n: int, delta: int):
    perm = np.empty(n, dtype=np.int32)
    lib().oracle_ntt_permutation(_p(perm, _i32p), n, delta)
    return perm


def _u32(values):
    return (ctypes.c_uint32 * len(values))(*values)


def chacha_block(seed, nonce, counter: int):
    out = (ctypes.c_uint32 * 16)()
    lib().oracle_chacha_block(_u32(seed), _u32(nonce), counter, out)
    return list(out)


def rand_int(seed, nonce, counter0: int, count: int, max_value: int, shift: int = 0):
    out = np.empty(count, dtype=np.int64)
    lib().oracle_rand_int(_u32(seed), _u32(nonce), counter0, count, max_value, shift, _p(out))
    return out


def discrete_gaussian(seed, nonce, counter0: int, count: int, tree):
    t = np.ascontiguousarray(np.asarray(tree, dtype=np.uint64))
    size = len(t) // 2
    depth = size.bit_length()
    out = np.empty(count, dtype=np.int64)
    lib().oracle_discrete_gaussian(_u32(seed), _u32(nonce), counter0, count, _p(t, _u64p), size,
                                   depth, _p(out))
    return out


class Context:
    """The oracle's view of one prime chain (all primes, specials last)."""

    def __init__(self, log_n: int, q, special_prime_count: int):
        self.log_n = log_n
        self.n = 1 << log_n
        self.q = np.ascontiguousarray(np.asarray(q, dtype=np.uint64))
        self.prime_count = len(self.q)
        self.special_prime_count = special_prime_count
        self.chain_count = self.prime_count - special_prime_count
        self._ctx = lib().oracle_ctx_new(log_n, self.prime_count, special_prime_count,
                                         _p(self.q, _u64p))

    def __del__(self):
        if getattr(self, "_ctx", None) and _lib is not None:
            _lib.oracle_ctx_free(self._ctx)
            self._ctx = None

    def tables(self):
        P, n = self.prime_count, self.n
        k = np.empty(P, dtype=np.uint64)
        r2 = np.empty(P, dtype=np.int64)
        ninv = np.empty(P, dtype=np.int64)
        root = np.empty((P, n - 1), dtype=np.int64)
        rinv = np.empty((P, n - 1), dtype=np.int64)
        lib().oracle_ctx_tables(self._ctx, _p(k, _u64p), _p(r2), _p(ninv), _p(root), _p(rinv))
        return dict(k=k, r_squared=r2, n_inverse=ninv, root=root, root_inverse=rinv)

    def chains(self, moduli_id: int) -> int:
        return self.chain_count - moduli_id

    def partition_count(self, moduli_id: int) -> int:
        return lib().oracle_partition_count(self._ctx, moduli_id)

    def to_ntt(self, moduli_id, x):
        x = np.ascontiguousarray(x, dtype=np.int64)
        y = np.empty_like(x)
        polys = x.shape[0] if x.ndim == 3 else 1
        chains = x.shape[-2]
        lib().oracle_to_ntt(self._ctx, moduli_id, chains, polys, _p(x), _p(y))
        return y

    def to_intt(self, moduli_id, x):
        x = np.ascontiguousarray(x, dtype=np.int64)
        y = np.empty_like(x)
        polys = x.shape[0] if x.ndim == 3 else 1
        chains = x.shape[-2]
        lib().oracle_to_intt(self._ctx, moduli_id, chains, polys, _p(x), _p(y))
        return y

    def tensor(self, moduli_id, a, b):
        a = np.ascontiguousarray(a, dtype=np.int64)
        b = np.ascontiguousarray(b, dtype=np.int64)
        L = self.chains(moduli_id)
        out = np.empty((3, L, self.n), dtype=np.int64)
        lib().oracle_tensor(self._ctx, moduli_id, _p(a), _p(b), _p(out))
        return out

    def relinearize(self, moduli_id, ct, key_moduli_id, key):
        ct = np.ascontiguousarray(ct, dtype=np.int64)
        key = np.ascontiguousarray(key, dtype=np.int64)
        L = self.chains(moduli_id)
        out = np.empty((2, L, self.n), dtype=np.int64)
        lib().oracle_relinearize(self._ctx, moduli_id, _p(ct), key_moduli_id, _p(key), _p(out))
        return out

    def key_switch(self, moduli_id, x, key_moduli_id, key):
        x = np.ascontiguousarray(x, dtype=np.int64)
        key = np.ascontiguousarray(key, dtype=np.int64)
        L = self.chains(moduli_id)
        out = np.empty((2, L, self.n), dtype=np.int64)
        lib().oracle_key_switch(self._ctx, moduli_id, _p(x), key_moduli_id, _p(key), _p(out))
        return out

    def mixed_radix(self, moduli_id, key_moduli_id, x):
        """rns_to_mrs (core_key_switch.cpp:21-56) of every partition of the
        coefficient-form polynomial x: each limb's digit at the limb's position (K > 1)."""
        x = np.ascontiguousarray(x, dtype=np.int64)
        out = np.empty((self.chains(moduli_id), self.n), dtype=np.int64)
        lib().oracle_mixed_radix(self._ctx, moduli_id, key_moduli_id, _p(x), _p(out))
        return out

    def mod_down(self, moduli_id, x):
        """mod_down (core_key_switch.cpp:110-160) of one NTT-form polynomial of all the
        primes at moduli_id: its chains(moduli_id) canonical coefficient-form limbs."""
        x = np.ascontiguousarray(x, dtype=np.int64)
        out = np.empty((self.chains(moduli_id), self.n), dtype=np.int64)
        lib().oracle_mod_down(self._ctx, moduli_id, _p(x), _p(out))
        return out

    def rescale(self, moduli_id, x):
        x = np.ascontiguousarray(x, dtype=np.int64)
        polys = x.shape[0]
        L = self.chains(moduli_id)
        y = np.empty((polys, L - 1, self.n), dtype=np.int64)
        lib().oracle_rescale(self._ctx, moduli_id, polys, _p(x), _p(y))
        return y

    def _ks_call(self, fn, moduli_id, ct, key_moduli_id, key, *extra):
        ct = np.ascontiguousarray(ct, dtype=np.int64)
        key = np.ascontiguousarray(key, dtype=np.int64)
        out = np.empty((2, self.chains(moduli_id), self.n), dtype=np.int64)
        fn(self._ctx, moduli_id, _p(ct), key_moduli_id, _p(key), *extra, _p(out))
        return out

    def switch_key(self, moduli_id, ct, key_moduli_id, key):
        return self._ks_call(lib().oracle_switch_key, moduli_id, ct, key_moduli_id, key)

    def conjugate(self, moduli_id, ct, key_moduli_id, key):
        return self._ks_call(lib().oracle_conjugate, moduli_id, ct, key_moduli_id, key)

    def rotate(self, moduli_id, ct, key_moduli_id, key, delta):
        return self._ks_call(lib().oracle_rotate, moduli_id, ct, key_moduli_id, key, delta)

    def deviations(self, scale: float, one_more_level: bool):
        out = np.empty(self.chain_count - 1, dtype=np.float64)
        lib().oracle_deviations(self._ctx, scale, int(one_more_level),
                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def level_down(self, x, source_level: int, level: int, rescaled: bool, scale: float,
                   one_more_level: bool):
        """Engine level_down of a coefficient-form (or rescaled) text."""
        x = np.ascontiguousarray(x, dtype=np.int64)
        full = self.chain_count - 2
        src_mid = full - source_level + (1 if rescaled else 0)
        dst_mid = full - level
        mult = np.zeros(self.chain_count, dtype=np.int64)
        lib().oracle_level_down_multiplier(self._ctx, scale, int(one_more_level), source_level,
                                           level, int(rescaled), _p(mult))
        y = np.empty((x.shape[0], self.chains(dst_mid), self.n), dtype=np.int64)
        lib().oracle_level_down(self._ctx, src_mid, x.shape[0], int(rescaled), dst_mid, _p(mult),
                                _p(x), _p(y))
        return y

    def encode(self, values, log_slot: int, level: int, scale_bits: int,
               include_special: bool = False, one_more_level: bool = True):
        """CKKSCore::encode of real (float) or complex slot values; returns
        (limbs [1][L][N], ckks_scale as a numpy longdouble)."""
        f64 = ctypes.POINTER(ctypes.c_double)
        scale = float(2 ** scale_bits)
        ckks = np.zeros(1, dtype=np.longdouble)  # x87 extended, as the C long double
        sbt = ctypes.c_double()
        flag = ctypes.c_int()
        first = ctypes.c_int()
        mult = np.zeros(self.prime_count, dtype=np.int64)
        lib().oracle_encode_level(self._ctx, scale, scale_bits, int(one_more_level), level,
                                  ckks.ctypes.data, ctypes.byref(sbt), ctypes.byref(flag),
                                  ctypes.byref(first), _p(mult))
        slot = 1 << log_slot
        v = np.asarray(values)
        re = np.zeros(slot)
        im = np.zeros(slot) if np.iscomplexobj(v) else None
        m = min(len(v), slot)
        re[:m] = np.real(v[:m])
        if im is not None:
            im[:m] = np.imag(v[:m])
        mid = self.chain_count - 2 - level
        limbs = self.prime_count - mid if include_special else self.chain_count - mid
        out = np.zeros((1, limbs, self.n), dtype=np.int64)
        lib().oracle_encode(self._ctx, re.ctypes.data_as(f64),
                            im.ctypes.data_as(f64) if im is not None else None, log_slot, sbt.value,
                            flag.value, first.value, _p(mult), limbs, _p(out))
        return out, ckks[0]

    def decode_plaintext(self, x, moduli_id: int, log_slot: int, ckks_scale, scale_bits: int,
                         complex_output: bool = True):
        """Engine decode of a coefficient-form plaintext [L][N] (rescale loop
        included); ckks_scale is a numpy longdouble."""
        x = np.ascontiguousarray(x, dtype=np.int64)
        f64 = ctypes.POINTER(ctypes.c_double)
        s = np.array([ckks_scale], dtype=np.longdouble)
        slot = 1 << log_slot
        re = np.zeros(slot)
        im = np.zeros(slot)
        lib().oracle_decode_plaintext(self._ctx, _p(x), moduli_id, log_slot, s.ctypes.data,
                                      float(2 ** scale_bits), re.ctypes.data_as(f64),
                                      im.ctypes.data_as(f64) if complex_output else None)
        return re + 1j * im if complex_output else re

    def rotate_plain(self, moduli_id, x, delta, ntt_form=False):
        x = np.ascontiguousarray(x, dtype=np.int64)
        y = np.empty_like(x)
        fn = lib().oracle_rotate_plain_ntt if ntt_form else lib().oracle_rotate_plain
        fn(self._ctx, moduli_id, x.shape[0], delta, _p(x), _p(y))
        return y

    def mult_relin_rescale(self, moduli_id, a, b, key_moduli_id, key):
        a = np.ascontiguousarray(a, dtype=np.int64)
        b = np.ascontiguousarray(b, dtype=np.int64)
        key = np.ascontiguousarray(key, dtype=np.int64)
        L = self.chains(moduli_id)
        out = np.empty((2, L - 2, self.n), dtype=np.int64)
        lib().oracle_mult_relin_rescale(self._ctx, moduli_id, _p(a), _p(b), key_moduli_id,
                                        _p(key), _p(out))
        return out
