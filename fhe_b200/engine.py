"""Python host mirror of the reference engine API over the C ABI.

Names and argument meaning follow DESILO FHE's CKKSEngine (src/ckks/engine.h):
``multiply``, ``relinearize``, ``rescale``, ``ntt`` / ``intt``; objects are HBM
resident and wrapped by :class:`Data`.  Errors raise :class:`FheError` carrying the
reference's message text (``"<Function Name>: <reason>"``).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import FheError, check  # noqa: F401  (re-exported)

# DataFlag (src/data/flag.h:7-13)
NONE, COMPLEX, NTT_FORM, RESCALED, SPARSE, INCLUDE_SPECIAL = 0, 1, 2, 4, 8, 16
# Object kinds (include/fhe_b200.h)
SECRET_KEY, PUBLIC_KEY, RELINEARIZATION_KEY, UNIT_CIPHERTEXT, UNIT_PLAINTEXT = 1, 2, 3, 4, 5
FIXED_ROTATION_KEY, CONJUGATION_KEY, KEY_SWITCHING_KEY = 6, 7, 8
# SchemePreset (src/engine/scheme_preset.h)
CKKS_40_60_DEFAULT, CKKS_54_60_BOOTSTRAP = 1, 2
CKKS_40_60_DEFAULT_ENGINE_TEST, CKKS_54_60_BOOTSTRAP_ENGINE_TEST = 3, 4


class Data:
    """One HBM-resident object (key, ciphertext or plaintext)."""

    def __init__(self, engine: "Engine", handle: ctypes.c_void_p):
        self.engine = engine
        self._h = handle

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        inf = _lib.FheDataInfo()
        check(_lib.load().fhe_data_info_get(self._h, ctypes.byref(inf)))
        return dict(type=inf.type, flag=inf.flag, moduli_id=inf.moduli_id, level=inf.level,
                    polys=inf.polys, chains=inf.chains, delta=inf.delta, scale=inf.ckks_scale)

    @property
    def level(self) -> int:
        return self.info()["level"]

    def download(self) -> np.ndarray:
        i = self.info()
        out = np.empty((i["polys"], i["chains"], self.engine.coeff_count), dtype=np.int64)
        check(_lib.load().fhe_data_download(self._h, out.ctypes.data_as(_lib._i64p)))
        return out

    def serialize(self) -> bytes:
        """The object in the engine's wire format (header and limbs)."""
        size = ctypes.c_uint64()
        check(_lib.load().fhe_data_serialized_size(self._h, ctypes.byref(size)))
        buf = ctypes.create_string_buffer(size.value)
        check(_lib.load().fhe_data_serialize(self._h, buf, size.value))
        return buf.raw

    def set_delta(self, delta: int) -> None:
        check(_lib.load().fhe_data_set_delta(self._h, delta))

    def device_pointer(self) -> int:
        p = _lib._i64p()
        check(_lib.load().fhe_data_device_pointer(self._h, ctypes.byref(p)))
        return ctypes.cast(p, ctypes.c_void_p).value

    def free(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().fhe_data_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class BootstrapKey:
    """A bootstrap key on the device (BootstrapKey, data/bootstrap.h:24-44)."""

    def __init__(self, engine: "Engine", handle):
        self.engine = engine
        self._h = handle

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        sc, shift, count = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        nbytes = ctypes.c_uint64()
        check(_lib.load().fhe_bootstrap_key_info(self._h, ctypes.byref(sc), ctypes.byref(shift),
                                                 ctypes.byref(count), ctypes.byref(nbytes)))
        return dict(stage_count=sc.value, inner_loop_shift=shift.value,
                    rotation_key_count=count.value, bytes=nbytes.value)

    def deltas(self) -> list:
        count = ctypes.c_int()
        check(_lib.load().fhe_bootstrap_key_deltas(self._h, None, 0, ctypes.byref(count)))
        arr = (ctypes.c_int * max(count.value, 1))()
        check(_lib.load().fhe_bootstrap_key_deltas(self._h, arr, count.value, ctypes.byref(count)))
        return list(arr[:count.value])

    def rotation_key(self, delta: int) -> Data:
        h = ctypes.c_void_p()
        check(_lib.load().fhe_bootstrap_key_rotation_key(self.engine.handle, self._h, delta,
                                                         ctypes.byref(h)))
        return Data(self.engine, h)

    def stage(self, to_slot: bool, stage: int) -> tuple:
        """(level, inner loop count, outer loop count) of a stage."""
        lv, inner, outer = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(_lib.load().fhe_bootstrap_key_stage(self._h, int(to_slot), stage, ctypes.byref(lv),
                                                  ctypes.byref(inner), ctypes.byref(outer)))
        return lv.value, inner.value, outer.value

    def diagonal(self, to_slot: bool, stage: int, outer: int, inner: int):
        h = ctypes.c_void_p()
        check(_lib.load().fhe_bootstrap_key_diagonal(self.engine.handle, self._h, int(to_slot),
                                                     stage, outer, inner, ctypes.byref(h)))
        return Data(self.engine, h) if h.value else None

    def small_bootstrap_key(self):
        a, b = ctypes.c_void_p(), ctypes.c_void_p()
        check(_lib.load().fhe_bootstrap_key_small(self.engine.handle, self._h, ctypes.byref(a),
                                                  ctypes.byref(b)))
        return Data(self.engine, a), Data(self.engine, b)

    def free(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().fhe_bootstrap_key_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Engine:
    """CKKS engine on one B200 (create_ckks_engine(CKKSConfig))."""

    def __init__(self, log_coeff_count: int = 14, special_prime_count: int = 1,
                 max_level: int = -1, scheme_preset: int = CKKS_40_60_DEFAULT,
                 log_slot_count: int = -1):
        lib = _lib.load()
        cfg = _lib.FheConfig(log_coeff_count, log_slot_count, special_prime_count, max_level,
                             scheme_preset)
        h = ctypes.c_void_p()
        check(lib.fhe_engine_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        inf = _lib.FheEngineInfo()
        check(lib.fhe_engine_info_get(self._h, ctypes.byref(inf)))
        self.coeff_count = inf.coeff_count
        self.slot_count = inf.slot_count
        self.chain_count = inf.chain_count
        self.prime_count = inf.prime_count
        self.special_prime_count = inf.special_prime_count
        self.full_level = inf.full_level
        self.max_level = inf.max_level
        self.max_key_switching_level = inf.max_key_switching_level
        self.scale_bit_length = inf.scale_bit_length
        q = (ctypes.c_uint64 * self.prime_count)()
        check(lib.fhe_engine_moduli(self._h, q, self.prime_count))
        self.moduli = np.array(list(q), dtype=np.uint64)

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().fhe_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # ------------------------------------------------------------- metadata --
    def moduli_id(self, level: int) -> int:
        out = ctypes.c_int()
        check(_lib.load().fhe_engine_moduli_id(self._h, level, ctypes.byref(out)))
        return out.value

    def chains(self, moduli_id: int, include_special: bool = False) -> int:
        return self.chain_count - moduli_id + (self.special_prime_count if include_special else 0)

    def partition_count(self, moduli_id: int) -> int:
        k = self.special_prime_count
        return (self.chains(moduli_id) + k - 1) // k

    def synchronize(self) -> None:
        check(_lib.load().fhe_engine_synchronize(self._h))

    def set_stream(self, cuda_stream: int | None) -> None:
        check(_lib.load().fhe_engine_set_stream(self._h, cuda_stream or None))

    # ----------------------------------------------------------- profiling --
    def set_profiling(self, enable: bool) -> None:
        check(_lib.load().fhe_engine_set_profiling(self._h, int(enable)))

    def profile(self) -> dict:
        """{kernel family: (launches, total device ms)} since the last reset."""
        buf = ctypes.create_string_buffer(1 << 16)
        check(_lib.load().fhe_engine_profile_report(self._h, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, launches, ms = line.split()
            out[name] = (int(launches), float(ms))
        return out

    def profile_reset(self) -> None:
        check(_lib.load().fhe_engine_profile_reset(self._h))

    @staticmethod
    def kernel_launch_count() -> int:
        return int(_lib.load().fhe_kernel_launch_count())

    # -------------------------------------------------------------- objects --
    def upload(self, limbs, moduli_id: int, flag: int = NONE, kind: int = UNIT_CIPHERTEXT,
               scale: float = 1.0) -> Data:
        limbs = np.ascontiguousarray(limbs, dtype=np.int64)
        polys = limbs.shape[0]
        chains = self.chains(moduli_id, bool(flag & INCLUDE_SPECIAL))
        if limbs.shape != (polys, chains, self.coeff_count):
            raise ValueError(f"limbs must have shape ({polys}, {chains}, {self.coeff_count})")
        h = ctypes.c_void_p()
        check(_lib.load().fhe_data_upload(self._h, kind, flag, moduli_id, polys, scale,
                                          limbs.ctypes.data_as(_lib._i64p), ctypes.byref(h)))
        return Data(self, h)

    def upload_from_pointer(self, host_ptr: int, moduli_id: int, polys: int, flag: int = NONE,
                            kind: int = UNIT_CIPHERTEXT, scale: float = 1.0) -> Data:
        """Upload limbs [polys][chains][N] from a raw host address (e.g. pinned memory)."""
        h = ctypes.c_void_p()
        check(_lib.load().fhe_data_upload(self._h, kind, flag, moduli_id, polys, scale,
                                          ctypes.cast(host_ptr, _lib._i64p), ctypes.byref(h)))
        return Data(self, h)

    def download_to_pointer(self, data: Data, host_ptr: int, wait: bool = True) -> None:
        fn = _lib.load().fhe_data_download if wait else _lib.load().fhe_data_download_async
        check(fn(data.handle, ctypes.cast(host_ptr, _lib._i64p)))

    def upload_relinearization_key(self, limbs, moduli_id: int) -> Data:
        return self.upload(limbs, moduli_id, NTT_FORM | INCLUDE_SPECIAL, RELINEARIZATION_KEY)

    def upload_fixed_rotation_key(self, limbs, moduli_id: int, delta: int) -> Data:
        """A FixedRotationKey: its key switching key limbs and its normalised delta."""
        key = self.upload(limbs, moduli_id, NTT_FORM | INCLUDE_SPECIAL, FIXED_ROTATION_KEY)
        key.set_delta(delta)
        return key

    def upload_conjugation_key(self, limbs, moduli_id: int) -> Data:
        return self.upload(limbs, moduli_id, NTT_FORM | INCLUDE_SPECIAL, CONJUGATION_KEY)

    def upload_key_switching_key(self, limbs, moduli_id: int) -> Data:
        return self.upload(limbs, moduli_id, NTT_FORM | INCLUDE_SPECIAL, KEY_SWITCHING_KEY)

    def _call(self, fn, *args) -> Data:
        h = ctypes.c_void_p()
        check(getattr(_lib.load(), fn)(self._h, *[a.handle for a in args], ctypes.byref(h)))
        return Data(self, h)

    # ------------------------------------------------------------ operations --
    def multiply(self, a: Data, b: Data, relinearization_key: Data | None = None) -> Data:
        if relinearization_key is None:
            return self._call("fhe_multiply", a, b)
        return self._call("fhe_multiply_relinearize", a, b, relinearization_key)

    def multiply_relinearize_rescale(self, a: Data, b: Data, relinearization_key: Data) -> Data:
        return self._call("fhe_multiply_relinearize_rescale", a, b, relinearization_key)

    def relinearize(self, ct: Data, relinearization_key: Data) -> Data:
        return self._call("fhe_relinearize", ct, relinearization_key)

    def rescale(self, ct: Data) -> Data:
        return self._call("fhe_rescale", ct)

    def ntt(self, text: Data) -> Data:
        return self._call("fhe_to_ntt", text)

    def intt(self, text: Data) -> Data:
        return self._call("fhe_to_intt", text)

    def level_down(self, text: Data, level: int) -> Data:
        h = ctypes.c_void_p()
        check(_lib.load().fhe_level_down(self._h, text.handle, level, ctypes.byref(h)))
        return Data(self, h)

    def rotate(self, ct: Data, key, delta: int | None = None,
               normalize_by_slot_count: bool = True) -> Data:
        """Rotate a ciphertext by one fixed rotation key, or by a list of fixed
        rotation keys (a RotationKey) and a delta; plaintexts rotate without a key."""
        if isinstance(key, (list, tuple)):
            arr = (ctypes.c_void_p * len(key))(*[k.handle for k in key])
            h = ctypes.c_void_p()
            check(_lib.load().fhe_rotate_with_keys(self._h, ct.handle, arr, len(key), delta,
                                                   int(normalize_by_slot_count), ctypes.byref(h)))
            return Data(self, h)
        if isinstance(key, BootstrapKey):
            h = ctypes.c_void_p()
            check(_lib.load().fhe_rotate_with_bootstrap_key(self._h, ct.handle, key.handle, delta,
                                                            ctypes.byref(h)))
            return Data(self, h)
        return self._call("fhe_rotate", ct, key)

    def rotate_batch(self, ct: Data, fixed_rotation_keys: list) -> list:
        """Hoisted rotations: one decomposition of ct for every fixed key."""
        n = len(fixed_rotation_keys)
        keys = (ctypes.c_void_p * n)(*[k.handle for k in fixed_rotation_keys])
        out = (ctypes.c_void_p * n)()
        check(_lib.load().fhe_rotate_batch(self._h, ct.handle, keys, n, out))
        return [Data(self, ctypes.c_void_p(out[i])) for i in range(n)]

    def rotate_plaintext(self, pt: Data, delta: int) -> Data:
        h = ctypes.c_void_p()
        check(_lib.load().fhe_rotate_plaintext(self._h, pt.handle, delta, ctypes.byref(h)))
        return Data(self, h)

    def conjugate(self, text: Data, conjugation_key: Data | None = None) -> Data:
        if conjugation_key is None:
            return self._call("fhe_conjugate_plaintext", text)
        return self._call("fhe_conjugate", text, conjugation_key)

    def encode(self, values, level: int | None = None, include_special: bool = False) -> Data:
        """encode_unit: real or complex slot values into a coefficient-form plaintext."""
        v = np.asarray(values)
        lvl = self.max_level if level is None else level
        h = ctypes.c_void_p()
        if np.iscomplexobj(v):
            re = np.ascontiguousarray(v.real, dtype=np.float64)
            im = np.ascontiguousarray(v.imag, dtype=np.float64)
            imp = im.ctypes.data_as(_lib._f64p)
        else:
            re = np.ascontiguousarray(v, dtype=np.float64)
            imp = None
        check(_lib.load().fhe_encode(self._h, re.ctypes.data_as(_lib._f64p), imp, re.size, lvl,
                                     int(include_special), ctypes.byref(h)))
        return Data(self, h)

    def decode(self, pt: Data, complex_output: bool = False) -> np.ndarray:
        """decode_unit (real parts) or decode_complex_unit_plaintext."""
        re = np.empty(self.slot_count, dtype=np.float64)
        im = np.empty(self.slot_count, dtype=np.float64) if complex_output else None
        check(_lib.load().fhe_decode(self._h, pt.handle, re.ctypes.data_as(_lib._f64p),
                                     im.ctypes.data_as(_lib._f64p) if im is not None else None))
        return re + 1j * im if complex_output else re

    # ------------------------------------------------------------ arithmetic --
    def add(self, a: Data, b) -> Data:
        """add(ct, ct | pt | float)."""
        if isinstance(b, (int, float)):
            return self._scalar("fhe_add_scalar", a, float(b))
        if b.info()["type"] == UNIT_PLAINTEXT:
            return self._call("fhe_add_plaintext", a, b)
        return self._call("fhe_add", a, b)

    def subtract(self, a, b) -> Data:
        """subtract(ct, ct | pt | float) or subtract(pt, ct)."""
        if isinstance(b, (int, float)):
            return self._scalar("fhe_subtract_scalar", a, float(b))
        if a.info()["type"] == UNIT_PLAINTEXT:
            return self._call("fhe_subtract_from_plaintext", a, b)
        if b.info()["type"] == UNIT_PLAINTEXT:
            return self._call("fhe_subtract_plaintext", a, b)
        return self._call("fhe_subtract", a, b)

    def multiply_plaintext(self, ct: Data, pt: Data) -> Data:
        return self._call("fhe_multiply_plaintext", ct, pt)

    def multiply_scalar(self, ct: Data, value: float) -> Data:
        return self._scalar("fhe_multiply_scalar", ct, float(value))

    def multiply_integer(self, ct: Data, value: int) -> Data:
        return self._scalar("fhe_multiply_integer", ct, int(value))

    def negate(self, ct: Data) -> Data:
        return self._call("fhe_negate", ct)

    def square(self, ct: Data, relinearization_key: Data | None = None) -> Data:
        h = ctypes.c_void_p()
        check(_lib.load().fhe_square(self._h, ct.handle,
                                     relinearization_key.handle if relinearization_key else None,
                                     ctypes.byref(h)))
        return Data(self, h)

    def _scalar(self, fn, ct: Data, value) -> Data:
        h = ctypes.c_void_p()
        check(getattr(_lib.load(), fn)(self._h, ct.handle, value, ctypes.byref(h)))
        return Data(self, h)

    # ------------------------------------------------------ keys, encryption --
    def seed(self, seed_words=None, nonce=None) -> None:
        """Reseed the engine's ChaCha20 stream (8 words, 2 nonce bytes; None: random)."""
        sw = (ctypes.c_uint32 * 8)(*seed_words) if seed_words is not None else None
        nn = (ctypes.c_uint8 * 2)(*nonce) if nonce is not None else None
        check(_lib.load().fhe_engine_seed(self._h, sw, nn))

    def _make(self, fn, *args) -> Data:
        h = ctypes.c_void_p()
        check(getattr(_lib.load(), fn)(self._h, *args, ctypes.byref(h)))
        return Data(self, h)

    def create_secret_key(self, level: int = -1, secret=None) -> Data:
        if secret is None:
            return self._make("fhe_create_secret_key", level)
        s = np.ascontiguousarray(secret, dtype=np.int64)
        return self._make("fhe_create_secret_key_from", s.ctypes.data_as(_lib._i64p), s.size, level)

    def create_sparse_secret_key(self, hamming_weight: int = 128, level: int = -1) -> Data:
        return self._make("fhe_create_sparse_secret_key", hamming_weight, level)

    def create_public_key(self, secret_key: Data, level: int = -1) -> Data:
        return self._make("fhe_create_public_key", secret_key.handle, level)

    def create_relinearization_key(self, secret_key: Data, level: int = -1) -> Data:
        return self._make("fhe_create_relinearization_key", secret_key.handle, level)

    def create_fixed_rotation_key(self, secret_key: Data, delta: int, level: int = -1,
                                  normalize_by_slot_count: bool = True) -> Data:
        return self._make("fhe_create_fixed_rotation_key", secret_key.handle, delta, level,
                          int(normalize_by_slot_count))

    def create_rotation_key(self, secret_key: Data, level: int = -1) -> list:
        arr = (ctypes.c_void_p * 64)()
        count = ctypes.c_int()
        check(_lib.load().fhe_create_rotation_keys(self._h, secret_key.handle, level, arr, 64,
                                                   ctypes.byref(count)))
        return [Data(self, ctypes.c_void_p(arr[i])) for i in range(count.value)]

    def create_conjugation_key(self, secret_key: Data, level: int = -1) -> Data:
        return self._make("fhe_create_conjugation_key", secret_key.handle, level)

    def encrypt(self, plaintext: Data, key: Data) -> Data:
        return self._call("fhe_encrypt", plaintext, key)

    def decrypt(self, ciphertext: Data, secret_key: Data) -> Data:
        return self._call("fhe_decrypt", ciphertext, secret_key)

    # --------------------------------------------------------- bootstrapping --
    def create_small_bootstrap_key(self, secret_key: Data):
        """Returns (to_sparse, to_dense) key switching keys."""
        a, b = ctypes.c_void_p(), ctypes.c_void_p()
        check(_lib.load().fhe_create_small_bootstrap_key(self._h, secret_key.handle,
                                                         ctypes.byref(a), ctypes.byref(b)))
        return Data(self, a), Data(self, b)

    def deserialize(self, blob: bytes) -> Data:
        """An object from Data.serialize of an engine with the same parameters."""
        h = ctypes.c_void_p()
        check(_lib.load().fhe_data_deserialize(self._h, blob, len(blob), ctypes.byref(h)))
        return Data(self, h)

    def set_tensor_cores(self, mode) -> None:
        """Where the base conversions run: False/0 CUDA cores, True/1 the INT8 tensor
        pipe, 2 (default) the tensor pipe where it measured faster (ModDown from 4
        special primes, ModUp from 4; with 1 also ModUp's and ModDown's NTTs at N = 2^16);
        same words."""
        check(_lib.load().fhe_engine_set_tensor_cores(self._h, int(mode)))

    def set_tensor_core_wait_limit(self, limit: int) -> None:
        """Diagnostics: polls per tensor-core MMA round before a kernel gives up and
        flags an error for the next synchronize (0: at once; negative: default)."""
        check(_lib.load().fhe_engine_set_tensor_core_wait_limit(self._h, int(limit)))

    def set_graphs(self, enable: bool) -> None:
        """CUDA-graph replay of bootstrap(ct, rk, ck, bootstrap_key) (default on)."""
        check(_lib.load().fhe_engine_set_graphs(self._h, int(enable)))

    def set_fused_bsgs(self, enable: bool) -> None:
        """The inner loop of a bootstrap key's linear transforms as one fused kernel
        (default on) or as per-rotation kernels; same words either way."""
        check(_lib.load().fhe_engine_set_fused_bsgs(self._h, int(enable)))

    def set_value_transforms(self, enable: bool) -> None:
        """Multiply-then-relinearize transforms its inputs and tensor value-only on the
        limbs that relinearization reads only modulo q (default on), or every limb with
        the reference's butterflies; same words either way."""
        check(_lib.load().fhe_engine_set_value_transforms(self._h, int(enable)))

    def multiply_rotate_batch(self, a: list, b: list, relinearization_key: Data,
                              rotation_keys: list) -> list:
        """[rotate(multiply_relinearize_rescale(a[i], b[i], rk), rotation_keys[i])]: one
        serving step, replayed as a CUDA graph after its first run."""
        n = len(a)
        arr = lambda xs: (ctypes.c_void_p * n)(*[x.handle for x in xs])
        out = (ctypes.c_void_p * n)()
        check(_lib.load().fhe_multiply_rotate_batch(self._h, n, arr(a), arr(b),
                                                    relinearization_key.handle,
                                                    arr(rotation_keys), out))
        return [Data(self, ctypes.c_void_p(out[i])) for i in range(n)]

    def multiply_relinearize_rescale_batch(self, a: list, b: list,
                                           relinearization_key: Data) -> list:
        """[multiply_relinearize_rescale(a[i], b[i], rk)], the items run concurrently
        on the engine's worker streams; the same words."""
        n = len(a)
        arr = lambda xs: (ctypes.c_void_p * n)(*[x.handle for x in xs])
        out = (ctypes.c_void_p * n)()
        check(_lib.load().fhe_multiply_relinearize_rescale_batch(
            self._h, n, arr(a), arr(b), relinearization_key.handle, out))
        return [Data(self, ctypes.c_void_p(out[i])) for i in range(n)]

    def bootstrap_batch(self, cts: list, relinearization_key: Data, conjugation_key: Data,
                        bootstrap_key: "BootstrapKey") -> list:
        """[bootstrap(ct, rk, ck, bootstrap_key) for ct in cts], concurrently."""
        n = len(cts)
        arr = (ctypes.c_void_p * n)(*[c.handle for c in cts])
        out = (ctypes.c_void_p * n)()
        check(_lib.load().fhe_bootstrap_batch(self._h, n, arr, relinearization_key.handle,
                                              conjugation_key.handle, bootstrap_key.handle, out))
        return [Data(self, ctypes.c_void_p(out[i])) for i in range(n)]

    def set_concurrency(self, streams: int) -> None:
        """Streams the items of a batch share (1 to 8, default 4); same words."""
        check(_lib.load().fhe_engine_set_concurrency(self._h, int(streams)))

    def graph_counts(self) -> tuple:
        """(captured bootstrap graphs held, input shapes whose capture failed)."""
        a, b = ctypes.c_int(), ctypes.c_int()
        check(_lib.load().fhe_engine_graph_counts(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def create_bootstrap_key(self, secret_key: Data, stage_count: int = 3,
                             size: str = "medium") -> BootstrapKey:
        h = ctypes.c_void_p()
        check(_lib.load().fhe_create_bootstrap_key(self._h, secret_key.handle, stage_count,
                                                   size.encode(), ctypes.byref(h)))
        return BootstrapKey(self, h)

    def bootstrap(self, ct: Data, relinearization_key: Data, conjugation_key: Data,
                  rotation_keys, small_bootstrap_key=None, stage_count: int = 3) -> Data:
        """bootstrap(ct, rk, ck, bootstrap_key) or bootstrap(ct, rk, ck, rotation key,
        small bootstrap key, stage_count), as the reference's two overloads."""
        if isinstance(rotation_keys, BootstrapKey):
            h = ctypes.c_void_p()
            check(_lib.load().fhe_bootstrap_with_key(self._h, ct.handle, relinearization_key.handle,
                                                     conjugation_key.handle, rotation_keys.handle,
                                                     ctypes.byref(h)))
            return Data(self, h)
        arr = (ctypes.c_void_p * len(rotation_keys))(*[k.handle for k in rotation_keys])
        to_sparse, to_dense = small_bootstrap_key
        h = ctypes.c_void_p()
        check(_lib.load().fhe_bootstrap(self._h, ct.handle, relinearization_key.handle,
                                        conjugation_key.handle, arr, len(rotation_keys),
                                        to_sparse.handle, to_dense.handle, stage_count,
                                        ctypes.byref(h)))
        return Data(self, h)

    def switch_key(self, ct: Data, key_switching_key: Data) -> Data:
        return self._call("fhe_switch_key", ct, key_switching_key)

    def ntt_limbs(self, device_ptr: int, moduli_id: int, chains: int, polys: int,
                  poly_stride: int, inverse: bool = False) -> None:
        """Plain per-limb NTT/iNTT (SingleProcessor::ntt/intt) on device memory, in place."""
        check(_lib.load().fhe_ntt_limbs(self._h, ctypes.cast(device_ptr, _lib._i64p), moduli_id,
                                        chains, polys, poly_stride, int(inverse)))

    def mont_mult_limbs(self, a_ptr: int, b_ptr: int, y_ptr: int, moduli_id: int, chains: int,
                        polys: int, poly_stride: int) -> None:
        """SingleProcessor::mont_mult on device memory: y = REDC(a * b) per word."""
        check(_lib.load().fhe_mont_mult_limbs(self._h, a_ptr, b_ptr, y_ptr, moduli_id, chains,
                                              polys, poly_stride))
