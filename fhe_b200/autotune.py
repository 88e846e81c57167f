"""NTT shape autotuner: ``python -m fhe_b200.autotune [--out PATH]`` on a B200.

For every transform size it times each valid two-pass shape (the split between the
strided and the contiguous pass, the sub-transforms per CTA of the strided pass and
the tile of the contiguous pass) on a batch of 24 limbs, forward and inverse, with
the engine's CUDA-event profiling; checks that the shape's words equal the default
shape's (every shape performs the same butterflies); and writes the fastest shape
per size to ``fhe_b200/ntt_tuning.json``, which the package installs when it loads
the library.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

from . import _lib
from .engine import Engine

SIZES = {  # log_n: engine configuration with at least 24 primes where possible
    14: dict(log_coeff_count=14, special_prime_count=1),
    15: dict(log_coeff_count=15, special_prime_count=2),
    16: dict(log_coeff_count=16, special_prime_count=10),
    17: dict(log_coeff_count=17, special_prime_count=6),
}


def candidates(log_n: int):
    for s_second in range(4, 12):
        s_first = log_n - s_second
        if not 4 <= s_first <= 11:
            continue
        for first_columns_log in range(1, 6):
            for second_tile_log in (11, 12, 13):
                yield s_second, first_columns_log, second_tile_log


def current(log_n: int):
    lib = _lib.load()
    v = [_lib.ctypes.c_int() for _ in range(3)]
    _lib.check(lib.fhe_ntt_tuning_get(log_n, *[_lib.ctypes.byref(x) for x in v]))
    return tuple(x.value for x in v)


def time_shape(e: Engine, ptr: int, mid: int, limbs: int, stride: int, reps: int) -> float:
    e.profile_reset()
    for _ in range(reps):
        e.ntt_limbs(ptr, mid, limbs, 1, stride, inverse=False)
        e.ntt_limbs(ptr, mid, limbs, 1, stride, inverse=True)
    e.synchronize()
    return e.profile()["ntt_limbs"][1] / reps


MIN_GAIN = 0.03  # a shape replaces the default only when it is this much faster


def tune(log_n: int, reps: int = 10):
    lib = _lib.load()
    e = Engine(**SIZES[log_n])
    n = e.coeff_count
    mid = max(0, e.chain_count - 24)  # the last (up to) 24 primes of the chain
    limbs = e.chain_count - mid
    rng = np.random.default_rng(log_n)
    limbs_data = np.stack([rng.integers(0, int(q), size=n, dtype=np.int64)
                           for q in e.moduli[mid:mid + limbs]])[None]
    default = current(log_n)
    ref = e.upload(limbs_data, mid)
    e.ntt_limbs(ref.device_pointer(), mid, limbs, 1, limbs * n, inverse=False)
    want = ref.download()
    work = e.upload(limbs_data, mid)
    e.set_profiling(True)
    results = []
    for shape in candidates(log_n):
        if lib.fhe_ntt_tuning_set(log_n, *shape) != 0:
            continue
        check = e.upload(limbs_data, mid)
        e.ntt_limbs(check.device_pointer(), mid, limbs, 1, limbs * n, inverse=False)
        if not np.array_equal(check.download(), want):
            raise RuntimeError(f"shape {shape} changed the words at log_n {log_n}")
        time_shape(e, work.device_pointer(), mid, limbs, limbs * n, 2)  # warm
        results.append((time_shape(e, work.device_pointer(), mid, limbs, limbs * n, reps), shape))
    e.set_profiling(False)
    _lib.check(lib.fhe_ntt_tuning_set(log_n, *default))
    default_ms = next(ms for ms, shape in results if shape == default)
    best_ms, best = min(results)
    e.close()
    out = dict(s_second=best[0], first_columns_log=best[1], second_tile_log=best[2],
               ms=best_ms, default_ms=default_ms, limbs=limbs, candidates=len(results))
    return choose(out, default)


def choose(entry: dict, default) -> dict:
    """Keeps the default shape unless the best one wins by MIN_GAIN (the plain
    transform the tuner times is lighter than the fused ones the engine runs)."""
    if entry["ms"] > (1.0 - MIN_GAIN) * entry["default_ms"]:
        entry = dict(entry, s_second=default[0], first_columns_log=default[1],
                     second_tile_log=default[2], kept_default=True)
    return entry


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=_lib.TUNING_PATH)
    ap.add_argument("--sizes", default="14,15,16,17")
    args = ap.parse_args(argv)
    table = {"ntt": {}, "note": "forward + inverse NTT of the given limbs, CUDA-event timed, "
                                 "best of all valid shapes; written by fhe_b200.autotune"}
    for log_n in (int(x) for x in args.sizes.split(",")):
        table["ntt"][str(log_n)] = tune(log_n)
        print(log_n, table["ntt"][str(log_n)], flush=True)
    with open(args.out + ".tmp", "w") as f:
        json.dump(table, f, indent=1)
    os.replace(args.out + ".tmp", args.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
