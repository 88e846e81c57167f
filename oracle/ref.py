"""ctypes bindings for the compiled reference (oracle/_ref/libdesilo_ref.so).

TEST INFRASTRUCTURE ONLY.  The library is the reference's own C++ sources built
by ``make -C oracle ref`` together with ref_harness.cpp.  It is optional: callers
use :func:`available` and skip when it is absent.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "libdesilo_ref.so")
_i64p = ctypes.POINTER(ctypes.c_int64)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_lib = None

# SchemePreset values (engine/scheme_preset.h)
CKKS_40_60_DEFAULT = 1
CKKS_54_60_BOOTSTRAP = 2
CKKS_40_60_DEFAULT_ENGINE_TEST = 3
CKKS_54_60_BOOTSTRAP_ENGINE_TEST = 4


def available() -> bool:
    return os.path.exists(_LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(_LIB_PATH)
        L = _lib
        vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        sig = {
            "ref_cached_primes": (ci, [ci, ci, _u64p, ci]),
            "ref_engine_new": (vp, [ci, ci, ci, ci, ci, ci]),
            "ref_engine_free": (None, [vp]),
            "ref_engine_seed": (None, [vp, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint8)]),
            "ref_engine_info": (None, [vp, ctypes.POINTER(ci)]),
            "ref_moduli_id": (ci, [vp, ci]),
            "ref_chain_count": (ci, [vp, ci, ci]),
            "ref_partition_count": (ci, [vp, ci, ci]),
            "ref_tables": (ci, [vp, _u64p, _u64p, _i64p, _i64p, _i64p, _i64p]),
            "ref_key_switch_tables": (None, [vp, _i64p, _i64p, _i64p]),
            "ref_text_new": (vp, [vp, ci, ci, ci, ci, ctypes.c_longdouble, _i64p]),
            "ref_key_new": (vp, [vp, ci, ci, ci, _i64p]),
            "ref_handle_free": (None, [vp]),
            "ref_rotation_key_new": (vp, [vp, ci, ci, ci, ci, _i64p]),
            "ref_core_rotate": (vp, [vp, vp, vp]),
            "ref_core_conjugate": (vp, [vp, vp, vp]),
            "ref_handle_info": (ctypes.c_longdouble, [vp, ctypes.POINTER(ci)]),
            "ref_handle_dump": (None, [vp, vp, _i64p]),
            "ref_create_secret_key": (vp, [vp, ci]),
            "ref_create_secret_key_from": (vp, [vp, _i64p, ci]),
            "ref_create_public_key": (vp, [vp, vp, ci]),
            "ref_create_relinearization_key": (vp, [vp, vp, ci]),
            "ref_create_fixed_rotation_key": (vp, [vp, vp, ci, ci]),
            "ref_create_conjugation_key": (vp, [vp, vp, ci]),
            "ref_core_to_ntt": (vp, [vp, vp]),
            "ref_core_to_intt": (vp, [vp, vp]),
            "ref_core_tensor": (vp, [vp, vp, vp]),
            "ref_core_relinearize": (vp, [vp, vp, vp]),
            "ref_core_rescale": (vp, [vp, vp]),
            "ref_core_switch_key": (vp, [vp, vp, vp]),
            "ref_engine_multiply": (vp, [vp, vp, vp, vp]),
            "ref_engine_relinearize": (vp, [vp, vp, vp]),
            "ref_engine_rescale": (vp, [vp, vp]),
            "ref_engine_rotate": (vp, [vp, vp, vp]),
            "ref_engine_conjugate": (vp, [vp, vp, vp]),
            "ref_engine_level_down": (vp, [vp, vp, ctypes.c_int]),
            "ref_last_error": (ctypes.c_char_p, []),
            "ref_bench_bootstrap": (ctypes.c_double, [ctypes.c_int]),
            "ref_bench_bootstrap_with_key": (ctypes.c_double, [ctypes.c_int]),
            "ref_create_bootstrap_key": (vp, [vp, vp, ctypes.c_int, ctypes.c_char_p]),
            "ref_bootstrap_key_delta_count": (ctypes.c_int, [vp]),
            "ref_bootstrap_key_get": (vp, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
            "ref_bootstrap_key_stage": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int,
                                                       ctypes.POINTER(ctypes.c_int)]),
            "ref_bootstrap_key_diagonal": (vp, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int]),
            "ref_bootstrap_key_small": (vp, [vp, ctypes.c_int]),
            "ref_engine_bootstrap_with_key": (vp, [vp, vp, vp, vp, vp]),
            "ref_create_rotation_key": (vp, [vp, vp, ctypes.c_int]),
            "ref_rotation_key_count": (ctypes.c_int, [vp]),
            "ref_rotation_key_get": (vp, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
            "ref_create_small_bootstrap_key": (vp, [vp, vp]),
            "ref_small_bootstrap_key_part": (vp, [vp, ctypes.c_int]),
            "ref_engine_bootstrap": (vp, [vp, vp, vp, vp, vp, vp, ctypes.c_int]),
            "ref_engine_arith": (vp, [vp, ctypes.c_int, vp, vp]),
            "ref_engine_scalar": (vp, [vp, ctypes.c_int, vp, ctypes.c_double, ctypes.c_longlong]),
            "ref_cdt_tree": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]),
            "ref_engine_decode_real": (ctypes.c_int, [vp, vp, ctypes.POINTER(ctypes.c_double)]),
            "ref_deviations": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int]),
            "ref_engine_rotate_plain": (vp, [vp, vp, ctypes.c_int]),
            "ref_engine_conjugate_plain": (vp, [vp, vp]),
            "ref_engine_rotate_keys": (vp, [vp, vp, ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int]),
            "ref_engine_encode": (vp, [vp, ctypes.POINTER(cd), ctypes.POINTER(cd), ci, ci]),
            "ref_engine_decode": (ci, [vp, vp, ctypes.POINTER(cd), ctypes.POINTER(cd)]),
            "ref_engine_encrypt": (vp, [vp, vp, vp]),
            "ref_engine_decrypt": (vp, [vp, vp, vp]),
            "ref_bench_mult_relin_rescale": (cd, [ci, ci, ci, ci, ci, ci, ctypes.POINTER(cd)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
    return _lib


def cached_primes(kind: int, n: int):
    out = np.zeros(256, dtype=np.uint64)
    cnt = lib().ref_cached_primes(kind, n, out.ctypes.data_as(_u64p), 256)
    return out[:cnt].copy()


class Handle:
    """A reference object (key, ciphertext, plaintext) owned by the harness."""

    def __init__(self, engine: "Engine", ptr):
        if not ptr:
            raise RuntimeError("reference call failed: " + lib().ref_last_error().decode())
        self.engine = engine
        self.ptr = ptr

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.ref_handle_free(self.ptr)
            self.ptr = None

    def info(self):
        info = (ctypes.c_int * 6)()
        scale = lib().ref_handle_info(self.ptr, info)
        kind, flag, moduli_id, level, polys, chains = list(info)
        return dict(kind=kind, flag=flag, moduli_id=moduli_id, level=level, polys=polys,
                    chains=chains, scale=scale)

    def limbs(self) -> np.ndarray:
        i = self.info()
        out = np.empty((i["polys"], i["chains"], self.engine.n), dtype=np.int64)
        lib().ref_handle_dump(self.engine.ptr, self.ptr, out.ctypes.data_as(_i64p))
        return out


class Engine:
    def __init__(self, log_n=14, special_prime_count=1, max_level=-1,
                 preset=CKKS_40_60_DEFAULT, log_slot=-1, threads=1):
        self.ptr = lib().ref_engine_new(log_n, log_slot, special_prime_count, max_level, preset,
                                        threads)
        if not self.ptr:
            raise ValueError("reference rejected the config")
        info = (ctypes.c_int * 10)()
        lib().ref_engine_info(self.ptr, info)
        (self.n, self.chain_count, self.prime_count, self.full_level, self.max_level,
         self.max_ks_level, self.slot_count, self.special_prime_count, self.scale_bits,
         self.one_more_level) = list(info)

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.ref_engine_free(self.ptr)
            self.ptr = None

    def seed(self, seed8, nonce2):
        s = (ctypes.c_uint32 * 8)(*seed8)
        n = (ctypes.c_uint8 * 2)(*nonce2)
        lib().ref_engine_seed(self.ptr, s, n)

    def moduli_id(self, level):
        return lib().ref_moduli_id(self.ptr, level)

    def chains(self, moduli_id, include_special=False):
        return lib().ref_chain_count(self.ptr, moduli_id, int(include_special))

    def partition_count(self, moduli_id, key_moduli_id):
        return lib().ref_partition_count(self.ptr, moduli_id, key_moduli_id)

    def tables(self):
        P, n = self.prime_count, self.n
        q = np.empty(P, dtype=np.uint64)
        k = np.empty(P, dtype=np.uint64)
        r2 = np.empty(P, dtype=np.int64)
        ninv = np.empty(P, dtype=np.int64)
        root = np.empty((P, n - 1), dtype=np.int64)
        rinv = np.empty((P, n - 1), dtype=np.int64)
        lib().ref_tables(self.ptr, q.ctypes.data_as(_u64p), k.ctypes.data_as(_u64p),
                         r2.ctypes.data_as(_i64p), ninv.ctypes.data_as(_i64p),
                         root.ctypes.data_as(_i64p), rinv.ctypes.data_as(_i64p))
        return dict(q=q, k=k, r_squared=r2, n_inverse=ninv, root=root, root_inverse=rinv)

    def text(self, limbs, moduli_id, flag=0, kind=4, scale=1.0):
        limbs = np.ascontiguousarray(limbs, dtype=np.int64)
        return Handle(self, lib().ref_text_new(self.ptr, kind, flag, moduli_id, limbs.shape[0],
                                               scale, limbs.ctypes.data_as(_i64p)))

    def relin_key(self, limbs, moduli_id):
        limbs = np.ascontiguousarray(limbs, dtype=np.int64)
        return Handle(self, lib().ref_key_new(self.ptr, 3, moduli_id, limbs.shape[0],
                                              limbs.ctypes.data_as(_i64p)))

    def switching_key(self, limbs, moduli_id):
        limbs = np.ascontiguousarray(limbs, dtype=np.int64)
        return Handle(self, lib().ref_key_new(self.ptr, 8, moduli_id, limbs.shape[0],
                                              limbs.ctypes.data_as(_i64p)))

    def fixed_rotation_key(self, limbs, moduli_id, delta):
        limbs = np.ascontiguousarray(limbs, dtype=np.int64)
        return Handle(self, lib().ref_rotation_key_new(self.ptr, 6, moduli_id, limbs.shape[0], delta,
                                                       limbs.ctypes.data_as(_i64p)))

    def conjugation_key(self, limbs, moduli_id):
        limbs = np.ascontiguousarray(limbs, dtype=np.int64)
        return Handle(self, lib().ref_rotation_key_new(self.ptr, 7, moduli_id, limbs.shape[0], -1,
                                                       limbs.ctypes.data_as(_i64p)))

    def core_rotate(self, ct, fixed_key):
        return self._h(lib().ref_core_rotate(self.ptr, ct.ptr, fixed_key.ptr))

    def core_conjugate(self, ct, ck):
        return self._h(lib().ref_core_conjugate(self.ptr, ct.ptr, ck.ptr))

    def _h(self, ptr):
        return Handle(self, ptr)

    # keys
    def create_secret_key(self, level=-1):
        return self._h(lib().ref_create_secret_key(self.ptr, level))

    def create_public_key(self, sk, level=-1):
        return self._h(lib().ref_create_public_key(self.ptr, sk.ptr, level))

    def create_relinearization_key(self, sk, level=-1):
        return self._h(lib().ref_create_relinearization_key(self.ptr, sk.ptr, level))

    def create_fixed_rotation_key(self, sk, delta, level=-1):
        return self._h(lib().ref_create_fixed_rotation_key(self.ptr, sk.ptr, delta, level))

    def create_conjugation_key(self, sk, level=-1):
        return self._h(lib().ref_create_conjugation_key(self.ptr, sk.ptr, level))

    # core ops
    def core_to_ntt(self, h):
        return self._h(lib().ref_core_to_ntt(self.ptr, h.ptr))

    def core_to_intt(self, h):
        return self._h(lib().ref_core_to_intt(self.ptr, h.ptr))

    def core_tensor(self, a, b):
        return self._h(lib().ref_core_tensor(self.ptr, a.ptr, b.ptr))

    def core_relinearize(self, ct, rk):
        return self._h(lib().ref_core_relinearize(self.ptr, ct.ptr, rk.ptr))

    def core_rescale(self, ct):
        return self._h(lib().ref_core_rescale(self.ptr, ct.ptr))

    def core_switch_key(self, ct, ksk):
        return self._h(lib().ref_core_switch_key(self.ptr, ct.ptr, ksk.ptr))

    # engine ops
    def multiply(self, a, b, rk=None):
        return self._h(lib().ref_engine_multiply(self.ptr, a.ptr, b.ptr, rk.ptr if rk else None))

    def relinearize(self, a, rk):
        return self._h(lib().ref_engine_relinearize(self.ptr, a.ptr, rk.ptr))

    def rescale(self, a):
        return self._h(lib().ref_engine_rescale(self.ptr, a.ptr))

    def rotate(self, a, fixed_key):
        return self._h(lib().ref_engine_rotate(self.ptr, a.ptr, fixed_key.ptr))

    def conjugate(self, a, ck=None):
        if ck is None:
            return self._h(lib().ref_engine_conjugate_plain(self.ptr, a.ptr))
        return self._h(lib().ref_engine_conjugate(self.ptr, a.ptr, ck.ptr))

    def deviations(self):
        out = np.zeros(256, dtype=np.float64)
        n = lib().ref_deviations(self.ptr, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 256)
        return out[:n]

    ARITH = dict(add=0, subtract=1, add_plain=2, subtract_plain=3, subtract_from_plain=4,
                 multiply_plain=5, negate=6, square=7, square_relinearize=8)
    SCALAR = dict(add_scalar=0, subtract_scalar=1, multiply_scalar=2, multiply_integer=3)

    def arith(self, op, a, b=None):
        return self._h(lib().ref_engine_arith(self.ptr, self.ARITH[op], a.ptr,
                                              b.ptr if b is not None else None))

    def scalar(self, op, a, value):
        return self._h(lib().ref_engine_scalar(self.ptr, self.SCALAR[op], a.ptr, float(value),
                                               int(value) if op == "multiply_integer" else 0))

    def create_rotation_key(self, sk, level=-1):
        """Returns (owner handle, [(fixed key view, delta), ...])."""
        owner = self._h(lib().ref_create_rotation_key(self.ptr, sk.ptr, level))
        views = []
        for i in range(lib().ref_rotation_key_count(owner.ptr)):
            d = ctypes.c_int()
            views.append((self._h(lib().ref_rotation_key_get(owner.ptr, i, ctypes.byref(d))),
                          d.value))
        return owner, views

    def create_small_bootstrap_key(self, sk):
        owner = self._h(lib().ref_create_small_bootstrap_key(self.ptr, sk.ptr))
        return owner, [self._h(lib().ref_small_bootstrap_key_part(owner.ptr, i)) for i in (0, 1)]

    def bootstrap(self, ct, rk, ck, rotk, sbk, stage_count):
        return self._h(lib().ref_engine_bootstrap(self.ptr, ct.ptr, rk.ptr, ck.ptr, rotk.ptr,
                                                  sbk.ptr, stage_count))

    def create_bootstrap_key(self, sk, stage_count, size="medium"):
        """Returns the owner handle of a BootstrapKey."""
        return self._h(lib().ref_create_bootstrap_key(self.ptr, sk.ptr, stage_count,
                                                      size.encode()))

    def bootstrap_key_rotation_keys(self, bk):
        """[(key switching key view, delta), ...] in ascending delta order."""
        out = []
        for i in range(lib().ref_bootstrap_key_delta_count(bk.ptr)):
            d = ctypes.c_int()
            out.append((self._h(lib().ref_bootstrap_key_get(bk.ptr, i, ctypes.byref(d))),
                        d.value))
        return out

    def bootstrap_key_stage(self, bk, to_slot, stage):
        """(level, inner loop count, outer loop count, process order entries)."""
        shape = (ctypes.c_int * 4)()
        if lib().ref_bootstrap_key_stage(bk.ptr, int(to_slot), stage, shape) != 0:
            raise IndexError(stage)
        return tuple(shape)

    def bootstrap_key_diagonal(self, bk, to_slot, stage, outer, inner):
        p = lib().ref_bootstrap_key_diagonal(bk.ptr, int(to_slot), stage, outer, inner)
        return self._h(p) if p else None

    def bootstrap_key_small(self, bk):
        return [self._h(lib().ref_bootstrap_key_small(bk.ptr, i)) for i in (0, 1)]

    def bootstrap_with_key(self, ct, rk, ck, bk):
        return self._h(lib().ref_engine_bootstrap_with_key(self.ptr, ct.ptr, rk.ptr, ck.ptr,
                                                           bk.ptr))

    def level_down(self, a, level):
        return self._h(lib().ref_engine_level_down(self.ptr, a.ptr, level))

    def rotate_plain(self, a, delta):
        return self._h(lib().ref_engine_rotate_plain(self.ptr, a.ptr, delta))

    def rotate_keys(self, a, fixed_keys, delta, by_slot_count=False):
        arr = (ctypes.c_void_p * len(fixed_keys))(*[k.ptr for k in fixed_keys])
        return self._h(lib().ref_engine_rotate_keys(self.ptr, a.ptr, arr, len(fixed_keys), delta,
                                                    int(by_slot_count)))

    def encode(self, values, level=-1, real=False):
        cd = ctypes.POINTER(ctypes.c_double)
        if real:
            re = np.ascontiguousarray(np.asarray(values, dtype=np.float64))
            return self._h(lib().ref_engine_encode(self.ptr, re.ctypes.data_as(cd), None,
                                                   len(re), level))
        values = np.asarray(values, dtype=np.complex128)
        re = np.ascontiguousarray(values.real)
        im = np.ascontiguousarray(values.imag)
        return self._h(lib().ref_engine_encode(self.ptr, re.ctypes.data_as(cd),
                                               im.ctypes.data_as(cd), len(values), level))

    def decode_real(self, pt):
        re = np.empty(self.slot_count)
        cd = ctypes.POINTER(ctypes.c_double)
        cnt = lib().ref_engine_decode_real(self.ptr, pt.ptr, re.ctypes.data_as(cd))
        return re[:cnt]

    def decode(self, pt):
        re = np.empty(self.slot_count)
        im = np.empty(self.slot_count)
        cd = ctypes.POINTER(ctypes.c_double)
        cnt = lib().ref_engine_decode(self.ptr, pt.ptr, re.ctypes.data_as(cd), im.ctypes.data_as(cd))
        return (re + 1j * im)[:cnt]

    def encrypt(self, pt, key):
        return self._h(lib().ref_engine_encrypt(self.ptr, pt.ptr, key.ptr))

    def decrypt(self, ct, sk):
        return self._h(lib().ref_engine_decrypt(self.ptr, ct.ptr, sk.ptr))


def bench_mult_relin_rescale(log_n, special_prime_count, level, threads, warmup, steps):
    times = (ctypes.c_double * max(steps, 1))()
    med = lib().ref_bench_mult_relin_rescale(log_n, special_prime_count, level, threads, warmup,
                                             steps, times)
    return med, list(times)[:steps]


def cdt_tree():
    """The reference sampler's CDT tree words."""
    out = (ctypes.c_uint64 * 256)()
    n = lib().ref_cdt_tree(out, 256)
    return [int(out[i]) for i in range(n)]


def bench_bootstrap(threads: int) -> float:
    """Milliseconds of one reference bootstrap (N = 2^16, 3 stages, all given threads)."""
    return float(lib().ref_bench_bootstrap(threads))


def bench_bootstrap_with_key(threads: int) -> float:
    """Milliseconds of one reference bootstrap with a medium 3-stage bootstrap key."""
    return float(lib().ref_bench_bootstrap_with_key(threads))
