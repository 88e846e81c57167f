"""Benchmark: CKKS HMult + relinearize + rescale throughput on B200.

Workload (one "step"): B independent pairs of fresh ciphertexts at N = 2^16 with 10
special primes, both at the maximum key-switching level (28 limbs), each pair going
through the reference's engine.multiply(a, b, relinearization_key) followed by
engine.rescale(.)  -- lazy rescale of both inputs to 27 limbs, NTT, tensor,
relinearize (hybrid key switching with dnum = 3 partitions [7, 10, 10]) and the
final rescale to 26 limbs.  Inputs are seeded uniform residues with a seeded random
relinearization key (operation time does not depend on the values).

  value : ciphertexts/s with inputs resident in HBM, device time (CUDA events on
          the engine's stream) over exactly K steps, max over ranks.
  e2e   : the same through the C ABI with pinned host buffers: every step uploads
          its inputs, runs the op and downloads the result.
  roofline : the dominant kernel family of the timed region, its algorithmic
          bytes per launch over its event-timed duration, against the measured
          HBM copy bandwidth (MEASURED_PEAKS.json).
  cpu_baseline : the reference's own CPU implementation (oracle/_ref, all host
          threads) on a bounded sample of the same operation.
  bootstrap : the other half of the headline metric, in the same run: ms per
          bootstrap at N = 2^16 (bootstrap preset, 2^15 slots, medium 3-stage
          bootstrap key, 8 ciphertexts per step), with precision bits, its own
          e2e, per-family kernel ms, clock record and reference CPU baseline.

Multi-GPU: replicas -- every rank runs the same per-GPU workload on its own GPU
with no data exchange ("scaling": "weak"); torch.distributed is used only for the
barrier and the max-over-ranks timing reduction.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B]
       python bench.py --impl reference ...
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, "tests", "golden"))

LOG_N = 16
SPECIAL = 10
METRIC = "HMult+relin+rescale ct/s at N=2^16 (K=10, dnum=3, 28-limb inputs)"
WORKLOAD = ("engine.multiply(ct_a, ct_b, relinearization_key) + engine.rescale, "
            "N=2^16, 10 special primes, inputs at level 26 (28 limbs), dnum=3")


# ----------------------------------------------------------------- helpers --

def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def aggregate(elapsed_ms: float, units: float, world: int, backend: str | None):
    """Max elapsed and summed units over ranks (identity on one process)."""
    if world <= 1 or backend is None:
        return elapsed_ms, units
    import torch
    import torch.distributed as dist

    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([elapsed_ms], dtype=torch.float64, device=dev)
    u = torch.tensor([units], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


def measured_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples the GPU's SM clock and throttle reasons during the timed region: through
    NVML in this process (initialised before the region starts, so each sample is
    one light query), else through nvidia-smi.  Rows keep nvidia-smi's CSV fields."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits: hw_slowdown, hw_thermal_slowdown,
    # sw_thermal_slowdown, sw_power_cap (the order of the rows' fields 5-8).
    REASON_BITS = (0x8, 0x40, 0x20, 0x4)

    def __init__(self, gpu_index: int, period_s: float = 0.05):
        self.gpu = gpu_index
        self.period = period_s
        self.rows = []
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None
        self._handle = None

    def _open_nvml(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            self._handle = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self._nvml = pynvml
        except Exception:
            self._nvml = None

    def _sample(self):
        try:
            if self._nvml is not None:
                m, h = self._nvml, self._handle
                sm = m.nvmlDeviceGetClockInfo(h, m.NVML_CLOCK_SM)
                mx = m.nvmlDeviceGetMaxClockInfo(h, m.NVML_CLOCK_SM)
                reasons = m.nvmlDeviceGetCurrentClocksEventReasons(h)
                power = m.nvmlDeviceGetPowerUsage(h) / 1000.0
                flags = ["Active" if reasons & bit else "Not Active" for bit in self.REASON_BITS]
                self.rows.append([str(self.gpu), str(sm), str(mx), f"{power:.1f}", hex(reasons)] + flags)
                return
            out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                  "--format=csv,noheader,nounits"], capture_output=True,
                                 text=True, timeout=5).stdout.strip()
            if out:
                self.rows.append([c.strip() for c in out.split(",")])
        except Exception:
            pass

    def _run(self):
        while not self._stop.wait(self.period if self._nvml is not None else 0.2):
            self._sample()

    def __enter__(self):
        self._open_nvml()
        if self._nvml is not None:
            self._sample()  # a first query before the region: NVML is warm when it starts
            self.rows.clear()
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=10)
        self._sample()  # the state at the end of the region
        if self._nvml is not None:
            try:
                self._nvml.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def kernel_bytes(L: int, E: int, dnum: int, n: int) -> dict:
    """Algorithmic HBM bytes per timed launch of each kernel family at the
    relinearize level (L limbs, E = L + K extended limbs): each limb operand read or
    written once, twiddle tables excluded.  Each partition's own L limbs of the
    extended polynomials are written by the tensor-product pass from the input's NTT
    form, so ModUp writes and transforms the other dnum * E - L.  The tensor's first
    two polynomials enter the key inner product as P d0, P d1 (the engine's default
    on this chain), so the tensor pass transforms the third alone and the ModDown
    epilogue adds nothing."""
    limb = 8 * n
    up = dnum * E - L
    return {
        "rescale": (2 * (L + 1) + 2 * L) * limb,          # 2 polys, L+1 -> L limbs
        "to_ntt": 2 * 4 * L * limb,                         # 4 polys in and out
        "rescale_to_ntt": (2 * (L + 1) + 2 * L) * limb,     # one input: rescaled, NTT
        "tensor_to_intt": (2 * L + L + L) * limb,           # a1, b1 in; d2 out, its own limbs
        "mixed_radix": 2 * L * limb,                        # digits of poly 2
        "mod_up_ntt": (L + up) * limb,                      # digits in, extended out
        "mod_up_contract_tc": (L + up) * limb,              # digits in, extended out
        "mod_up_ntt_tc": 2 * up * limb,                     # extended limbs in and out
        # ext + 2 key polys + the 4 NTT-form factors in, 2 out
        "key_inner_product": (3 * dnum * E + 4 * L + 2 * E) * limb,
        "mod_down_intt": 2 * 2 * E * limb,                  # 2 polys in and out
        "mod_down_epilogue": (2 * E + 2 * (L - 1)) * limb,
        "mod_down_epilogue_tc": (2 * E + 2 * (L - 1)) * limb,
    }


# ------------------------------------------------------------- reference arm --

INT8_NOMINAL_OPS = 4.5e15  # B200 dense INT8 tensor throughput, nominal (no measured figure)


def partition_sizes(L: int, K: int) -> list:
    """Limbs of each key-switching partition at L limbs (ckks/parameters.cpp:334-360)."""
    pc = (L + K - 1) // K
    return [min(L, s + K) - max(0, s) for s in range(L - pc * K, L, K)]


def pipe_figures(prof: dict, steps: int, pairs: int, n: int, L: int, K: int, sm_mhz, sms: int):
    """What bounds the headline step: butterflies per SM per clock of the transform
    families (their loaders and storers included) from the event-timed launches and
    the SM clock sampled during the run, and the INT8 operations the two tensor-core
    kernels issue per second against the nominal dense INT8 peak."""
    E = L + K
    dnum = (L + K - 1) // K
    hz = (sm_mhz or 1965.0) * 1e6
    log_n = n.bit_length() - 1
    bfly_per_limb = (n // 2) * log_n
    # ModUp transforms every extended limb but each partition's own (L in all), whose
    # NTT-form words the tensor's loader provides; the tensor pass transforms its
    # third polynomial alone (the first two enter the key inner product).
    transforms = {"rescale_to_ntt": 4 * L, "tensor_to_intt": L, "mod_up_ntt_tc": dnum * E - L,
                  "mod_down_intt": 2 * E}
    integer = {}
    for fam, limbs in transforms.items():
        if fam in prof:
            sec = prof[fam][1] / 1e3
            integer[fam] = {"limb_transforms_per_pair": limbs,
                            "butterflies_per_sm_per_clock":
                                pairs * steps * limbs * bfly_per_limb / (sec * sms * hz)}
    tiles = n // 128
    kb_down = (9 * K + 31) // 32 * 32
    issued = {
        # 2 polys x ceil(L/8) rounds of 128 x 128 x kb per 128 coefficients
        "mod_down_epilogue_tc": 2 * tiles * -(-L // 8) * 2 * 128 * 128 * kb_down,
        "mod_up_contract_tc": sum(tiles * -(-E // 8) * 2 * 128 * 128 * ((8 * a + 31) // 32 * 32)
                                  for a in partition_sizes(L, K)),
    }
    useful = {  # 64 byte-pair products per 64-bit multiply-accumulate
        "mod_down_epilogue_tc": 2 * 64 * 2 * n * K * L,
        "mod_up_contract_tc": 2 * 64 * n * sum(a * E for a in partition_sizes(L, K)),
    }
    tensor = {}
    for fam, ops in issued.items():
        if fam in prof:
            cnt, ms = prof[fam]
            sec = ms / cnt / 1e3
            tensor[fam] = {"issued_int8_ops_per_launch": ops,
                           "algorithmic_int8_ops_per_launch": useful[fam],
                           "avg_launch_ms": ms / cnt, "issued_ops_per_s": ops / sec,
                           "peak_ops_per_s": INT8_NOMINAL_OPS, "peak_source": "nominal",
                           "frac": ops / sec / INT8_NOMINAL_OPS}
    return integer, tensor


def run_reference(args, rank: int):
    """The reference's own CPU implementation of the path (oracle/_ref), all host
    threads; each step is one HMult+relin+rescale on the same config."""
    if rank != 0:
        return 0
    from oracle import ref

    threads = os.cpu_count() or 1
    line = {"impl": "reference", "metric": METRIC, "unit": "ct/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded uniform complex slots, fresh keys)",
            "config": {"workload": WORKLOAD, "threads": threads}}
    if not ref.available():
        from oracle import oracle
        import numpy as np
        from inputs import case_inputs

        # The compiled reference is absent: time the C restatement (single thread).
        from fhe_b200 import _lib
        import ctypes

        cfg = _lib.FheConfig(LOG_N, -1, SPECIAL, -1, 1)
        info = _lib.FheEngineInfo()
        qbuf = (ctypes.c_uint64 * 64)()
        _lib.check(_lib.load().fhe_parameters_query(ctypes.byref(cfg), ctypes.byref(info), qbuf, 64))
        q = np.array(qbuf[: info.prime_count], dtype=np.uint64)
        ctx = oracle.Context(LOG_N, q, SPECIAL)
        mid = info.chain_count - 2 - info.max_key_switching_level
        a, b, _, key = case_inputs(5, q, 1 << LOG_N, mid, SPECIAL)
        times = []
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            ctx.mult_relin_rescale(mid, a, b, mid, key)
            if i >= args.warmup:
                times.append((time.perf_counter() - t0) * 1e3)
        kind, cores = "port", 1
    else:
        _, times = ref.bench_mult_relin_rescale(LOG_N, SPECIAL, -1, threads, args.warmup, args.steps)
        kind, cores = "reference", threads
    ms = sum(times) / len(times)
    value = 1000.0 / ms
    line.update({"value": value, "ms_per_step": ms,
                 "cpu_baseline": {"value": value, "unit": "ct/s", "cores": cores, "kind": kind,
                                  "sample": f"{args.steps} ops after {args.warmup} warm-up"},
                 "e2e": {"value": value, "unit": "ct/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_sample():
    """Bounded CPU sample for the headline line (rank 0, one GPU only)."""
    try:
        from oracle import ref

        if ref.available():
            threads = os.cpu_count() or 1
            _, times = ref.bench_mult_relin_rescale(LOG_N, SPECIAL, -1, threads, 2, 10)
            ms = sum(times) / len(times)
            # The same operation on one host thread, a shorter sample.
            _, times1 = ref.bench_mult_relin_rescale(LOG_N, SPECIAL, -1, 1, 1, 3)
            ms1 = sum(times1) / len(times1)
            return {"value": 1000.0 / ms, "unit": "ct/s", "cores": threads, "kind": "reference",
                    "sample": "10 HMult+relin+rescale ops (after 2 warm-up) through the reference "
                              "CKKSEngine with CPU_PARALLEL, keygen excluded",
                    "single_thread": {"value": 1000.0 / ms1, "unit": "ct/s", "cores": 1,
                                      "sample": "3 ops (after 1 warm-up) on one thread"}}
    except Exception as exc:  # the baseline must not sink the GPU line
        return {"value": None, "unit": "ct/s", "cores": 0, "kind": "reference",
                "sample": f"failed: {exc}"}
    return {"value": None, "unit": "ct/s", "cores": 0, "kind": "port",
            "sample": "reference library not built on this host"}


# ------------------------------------------------------------ NTT microbench --

def run_ntt_microbench(args, torch, np, rank, world, local, backend, stream):
    """Forward NTT (SingleProcessor::ntt per limb) of `batch` polynomials of 24 limbs
    at N = 2^16 over the first 24 primes of the Gold chain, in place.  Algorithmic
    bytes: one read and one write of every limb (twiddles excluded)."""
    from fhe_b200 import Engine, UNIT_PLAINTEXT
    from inputs import uniform_limbs

    eng = Engine(log_coeff_count=16, special_prime_count=4)
    eng.set_stream(stream.cuda_stream)
    eng.set_concurrency(CONCURRENCY)
    n, limbs, B = eng.coeff_count, 24, args.batch
    rng = np.random.default_rng(5 + rank)
    buf = eng.upload(uniform_limbs(rng, eng.moduli[:limbs], B, n), eng.chain_count - limbs,
                     kind=UNIT_PLAINTEXT)
    ptr = buf.device_pointer()
    stride = limbs * n
    for _ in range(args.warmup):
        eng.ntt_limbs(ptr, 0, limbs, B, stride)
    torch.cuda.synchronize()
    if backend:
        torch.distributed.barrier()
    launches0 = Engine.kernel_launch_count()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            eng.ntt_limbs(ptr, 0, limbs, B, stride)
        stop.record(stream)
        torch.cuda.synchronize()
    elapsed = start.elapsed_time(stop)
    launches = Engine.kernel_launch_count() - launches0
    elapsed_max, units = aggregate(elapsed, float(B * args.steps), world, backend)
    bytes_per_step = 2 * B * limbs * n * 8
    gbs = bytes_per_step * args.steps * world / (elapsed_max / 1e3) / 1e9
    peak, peak_kind = measured_peaks()

    def timed_op(fn, nbytes):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(args.steps):
            fn()
        s1.record(stream)
        torch.cuda.synchronize()
        ms, u = aggregate(s0.elapsed_time(s1), float(B * args.steps), world, backend)
        return {"polys_per_s": u / (ms / 1e3),
                "achieved_gbs": nbytes * args.steps / (ms / 1e3) / 1e9,
                "frac_of_peak": nbytes * args.steps / (ms / 1e3) / 1e9 / peak}

    # The inverse transform, and SingleProcessor::mont_mult of two batches (config B's
    # pointwise product: reads a and b, writes y).
    other = eng.upload(uniform_limbs(rng, eng.moduli[:limbs], B, n), eng.chain_count - limbs,
                       kind=UNIT_PLAINTEXT)
    optr = other.device_pointer()
    extra = {
        "inverse_ntt": timed_op(lambda: eng.ntt_limbs(ptr, 0, limbs, B, stride, inverse=True),
                                bytes_per_step),
        "pointwise_mont_mult": timed_op(
            lambda: eng.mont_mult_limbs(optr, ptr, optr, 0, limbs, B, stride),
            3 * B * limbs * n * 8),
    }
    other.free()
    if rank == 0:
        print(json.dumps({
            "metric": "forward NTT polys/s (24 limbs, N=2^16)", "value": units / (elapsed_max / 1e3),
            "unit": "polys/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic uniform residues",
            "config": {"workload": "ntt 24 limbs x batch", "batch": B,
                       "l2": f"limbs larger than L2 for batch >= 11 ({B * limbs * n * 8 / 1e6:.0f} MB)"},
            "other_kernels": extra,
            "roofline": {"bound": "hbm", "achieved": gbs / world, "peak": peak, "unit": "GB/s",
                         "frac": gbs / world / peak, "traffic": None, "peak_source": peak_kind},
            "gpu_launches": launches, "clocks": clocks.summary()}), flush=True)
    buf.free()
    eng.close()
    return 0


# -------------------------------------------------------------- bootstrap --

CONCURRENCY = 4  # worker streams of batch calls (the engine's default; --streams)


BOOTSTRAP_BATCH = 8  # ciphertexts per step of the bootstrap measurement


def run_bootstrap_bench(args, torch, np, rank, world, local, backend, stream):
    """The bootstrap workloads as their own bench line."""
    line = bootstrap_measure(args, torch, np, rank, world, local, backend, stream,
                             args.workload == "bootstrap", args.batch)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def bootstrap_measure(args, torch, np, rank, world, local, backend, stream, with_key, B):
    """Bootstrapping at N = 2^16 (bootstrap preset, 4 special primes, 2^15 complex
    slots uniform in [-1, 1], 3 stages): each step bootstraps B ciphertexts
    encrypted at level 3.  Keys are made on the device before timing.  with_key: a
    "medium" bootstrap key (hoisted baby-step giant-step transforms); otherwise the
    rotation key and small bootstrap key.  Returns the bench line (every rank)."""
    from fhe_b200 import Engine
    from inputs import codec_values

    eng = Engine(log_coeff_count=16, special_prime_count=4, scheme_preset=2)
    eng.set_stream(stream.cuda_stream)
    eng.set_concurrency(CONCURRENCY)
    eng.set_tensor_cores(args.tensor_cores)
    eng.seed([11 + rank, 22, 33, 44, 55, 66, 77, 88], [1, 2])
    sk = eng.create_secret_key()
    rk = eng.create_relinearization_key(sk)
    ck = eng.create_conjugation_key(sk)
    if with_key:
        bk = eng.create_bootstrap_key(sk, 3, "medium")
        key_bytes = bk.info()["bytes"]
    else:
        rot = eng.create_rotation_key(sk)
        sbk = eng.create_small_bootstrap_key(sk)
        key_bytes = None
    values = [codec_values(100 + i, eng.slot_count, True) for i in range(B)]
    cts = [eng.encrypt(eng.encode(v, 3), sk) for v in values]

    def boot(c):
        if with_key:
            return eng.bootstrap(c, rk, ck, bk)
        return eng.bootstrap(c, rk, ck, rot, sbk, 3)

    def step(inputs):
        if with_key:  # one batch call: the bootstraps share the engine's worker streams
            return eng.bootstrap_batch(inputs, rk, ck, bk)
        return [boot(c) for c in inputs]

    for _ in range(args.warmup):
        step(cts)
    torch.cuda.synchronize()
    if backend:
        torch.distributed.barrier()
    launches0 = Engine.kernel_launch_count()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            outs = step(cts)
        stop.record(stream)
        torch.cuda.synchronize()
    elapsed = start.elapsed_time(stop)
    launches = Engine.kernel_launch_count() - launches0
    elapsed_max, units = aggregate(elapsed, float(B * args.steps), world, backend)
    ms_per_bootstrap = elapsed_max / (args.steps * B)
    # Precision of one output against the input slots (float64 oracle = the values).
    dec = eng.decode(eng.decrypt(outs[0], sk), complex_output=True)
    err = float(np.max(np.abs(dec - values[0])))
    bits = float(-np.log2(err)) if err > 0 else 64.0
    # Per-family device time of one bootstrap.
    eng.set_profiling(True)
    eng.profile_reset()
    step(cts[:1])
    families = {k: v[1] for k, v in eng.profile().items()}
    eng.set_profiling(False)
    # End to end: ciphertext limbs from pinned host memory, bootstrap, result back.
    host_ct = [torch.from_numpy(c.download()).pin_memory() for c in cts]
    out_host = torch.empty(tuple(outs[0].download().shape), dtype=torch.int64).pin_memory()
    info = cts[0].info()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ins = [eng.upload_from_pointer(h.data_ptr(), info["moduli_id"], 2, info["flag"],
                                       scale=float(info["scale"])) for h in host_ct]
        for o in step(ins):
            eng.download_to_pointer(o, out_host.data_ptr(), wait=False)
    eng.synchronize()  # the last results are in host memory
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = aggregate(e0.elapsed_time(e1), 0.0, world, backend)[0] / (args.steps * B)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import ref

            if ref.available():
                threads = os.cpu_count() or 1
                ms = (ref.bench_bootstrap_with_key if with_key else ref.bench_bootstrap)(threads)
                kind = "medium bootstrap key" if with_key else "rotation key"
                cpu = {"value": ms, "unit": "ms/bootstrap", "cores": threads, "kind": "reference",
                       "sample": f"1 bootstrap (N=2^16, 3 stages, {kind}) through the "
                                 "reference CKKSEngine with CPU_PARALLEL, keygen excluded"}
        except Exception as exc:
            cpu = {"value": None, "unit": "ms/bootstrap", "cores": 0, "kind": "reference",
                   "sample": f"failed: {exc}"}
    line = {
            "metric": "bootstrap ms at N=2^16 (2^15 slots, 3 stages)", "value": ms_per_bootstrap,
            "unit": "ms/bootstrap", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed_max / args.steps, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded uniform complex slots in [-1, 1], keys made on the device)",
            "config": {"workload": ("engine.bootstrap(ct, rk, ck, medium bootstrap key of 3 "
                                    "stages)" if with_key else
                                    "engine.bootstrap(ct, rk, ck, rotation key, small bootstrap "
                                    "key, 3)") + ", bootstrap preset, N=2^16, K=4, input level 3",
                       "ciphertexts_per_step": B, "precision_bits": bits,
                       "tensor_cores": ["off", "on", "auto"][args.tensor_cores],
                       "api": "fhe_bootstrap_batch" if with_key else "fhe_bootstrap",
                       "streams": CONCURRENCY if with_key else 1,
                       "bootstrap_key_bytes": key_bytes,
                       "cuda_graphs": {"captured": eng.graph_counts()[0],
                                       "capture_failed": eng.graph_counts()[1]},
                       "kernel_ms_per_bootstrap": families},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_ms, "unit": "ms/bootstrap",
                    "h2d_bytes_per_step": int(sum(h.numel() * 8 for h in host_ct)),
                    "d2h_bytes_per_step": int(out_host.numel() * 8 * B)},
            "gpu_launches": launches, "clocks": clocks.summary()}
    del outs, cts
    eng.close()
    return line


def run_batched_bench(args, torch, np, rank, world, local, backend, stream):
    """The batched uneven serving step at N = 2^16, K = 10: `batch` ciphertext pairs at
    levels uniform in 2..24, each multiplied, relinearized and rescaled, then rotated
    by 2^k with k uniform in 0..14 (one fixed rotation key per k, 1.8 GB resident),
    the whole batch replayed as one CUDA graph.  Per-operation latencies come from a
    direct (unreplayed) pass that times every item with its own events."""
    from fhe_b200 import Engine, NTT_FORM, INCLUDE_SPECIAL, RELINEARIZATION_KEY
    from inputs import uniform_limbs

    eng = Engine(log_coeff_count=LOG_N, special_prime_count=SPECIAL)
    eng.set_stream(stream.cuda_stream)
    eng.set_concurrency(CONCURRENCY)
    n = eng.coeff_count
    top = eng.moduli_id(eng.max_key_switching_level)
    rng = np.random.default_rng(77 + rank)
    parts = 2 * eng.partition_count(top)
    rk = eng.upload(uniform_limbs(rng, eng.moduli[top:], parts, n), top,
                    NTT_FORM | INCLUDE_SPECIAL, RELINEARIZATION_KEY)
    rot = [eng.upload_fixed_rotation_key(uniform_limbs(rng, eng.moduli[top:], parts, n), top, 1 << k)
           for k in range(15)]
    B = args.batch
    levels = rng.integers(2, 25, size=B)
    steps_k = rng.integers(0, 15, size=B)
    A, Bs, keys, host = [], [], [], []
    for lv, k in zip(levels, steps_k):
        mid = eng.moduli_id(int(lv))
        q = eng.moduli[mid:eng.chain_count]
        a, b = uniform_limbs(rng, q, 2, n), uniform_limbs(rng, q, 2, n)
        A.append(eng.upload(a, mid))
        Bs.append(eng.upload(b, mid))
        keys.append(rot[int(k)])
        host.append((mid, torch.from_numpy(a.reshape(-1)).pin_memory(),
                     torch.from_numpy(b.reshape(-1)).pin_memory()))

    def step():
        for o in eng.multiply_rotate_batch(A, Bs, rk, keys):
            o.free()

    for _ in range(max(args.warmup, 2)):  # direct run, then the capture
        step()
    torch.cuda.synchronize()
    if backend:
        torch.distributed.barrier()
    launches0 = Engine.kernel_launch_count()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            step()
        stop.record(stream)
        torch.cuda.synchronize()
    launches = Engine.kernel_launch_count() - launches0
    elapsed_max, units = aggregate(start.elapsed_time(stop), float(B * args.steps), world, backend)
    value = units / (elapsed_max / 1e3)

    # Per-operation latency: every item alone, direct, event-timed.
    eng.set_graphs(False)
    lat = []
    for a, b, k in zip(A, Bs, keys):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = eng.rotate(eng.multiply_relinearize_rescale(a, b, rk), k)
        e1.record(stream)
        torch.cuda.synchronize()
        lat.append(e0.elapsed_time(e1))
        out.free()
    eng.set_graphs(True)
    lat.sort()
    pct = lambda p: lat[min(len(lat) - 1, int(round(p / 100 * (len(lat) - 1))))]

    # End to end: every pair from pinned host memory, the batch, every result back.
    out_shapes = [o.download().size for o in eng.multiply_rotate_batch(A, Bs, rk, keys)]
    pin_out = [torch.empty(sz, dtype=torch.int64).pin_memory() for sz in out_shapes]

    def e2e_step():
        ins = []
        for mid, ha, hb in host:
            ins.append((eng.upload_from_pointer(ha.data_ptr(), mid, 2),
                        eng.upload_from_pointer(hb.data_ptr(), mid, 2)))
        outs = eng.multiply_rotate_batch([x[0] for x in ins], [x[1] for x in ins], rk, keys)
        for o, p in zip(outs, pin_out):
            eng.download_to_pointer(o, p.data_ptr(), wait=False)
        # No wait: the next step's uploads overlap this step's kernels; every object
        # is freed behind the work that reads it.

    e2e_step()
    e2e_step()
    eng.synchronize()
    torch.cuda.synchronize()
    e_steps = max(1, min(args.steps, 3))
    s2, t2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(e_steps):
        e2e_step()
    eng.synchronize()  # the last results are in host memory
    t2.record(stream)
    torch.cuda.synchronize()
    e_ms, e_units = aggregate(s2.elapsed_time(t2), float(B * e_steps), world, backend)
    if rank == 0:
        print(json.dumps({
            "metric": "batched uneven HMult+relin+rescale+rotate ct/s at N=2^16 (K=10)",
            "value": value, "unit": "ct/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 2), "ms_per_step": elapsed_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded uniform residues, random relinearization and rotation keys)",
            "config": {"workload": "engine.multiply_rotate_batch: per item multiply-relinearize-"
                                   "rescale then rotate by 2^k, levels uniform in 2..24, k "
                                   "uniform in 0..14, one CUDA graph per batch",
                       "batch": B, "log_n": LOG_N, "special_prime_count": SPECIAL,
                       "mean_input_limbs": float(np.mean(levels + 2)),
                       "l2": "inputs larger than L2",
                       "cuda_graphs": {"captured": eng.graph_counts()[0],
                                       "capture_failed": eng.graph_counts()[1]},
                       "latency_ms": {"p50": pct(50), "p99": pct(99), "mean": sum(lat) / len(lat),
                                      "note": "one item alone, direct launches, event-timed"}},
            "cpu_baseline": None,
            "e2e": {"value": e_units / (e_ms / 1e3), "unit": "ct/s",
                    "h2d_bytes_per_step": int(sum(h[1].numel() + h[2].numel() for h in host) * 8),
                    "d2h_bytes_per_step": int(sum(out_shapes) * 8)},
            "gpu_launches": launches, "clocks": clocks.summary()}), flush=True)
    eng.close()
    return 0


def run_plain_bench(args, torch, np, rank, world, local, backend, stream):
    """The plain CKKS pipeline of the reference's default engine (N = 2^14, one
    special prime, scale 2^40): per pair, encode two vectors of 2^13 complex slots,
    encrypt them with the public key, multiply and relinearize, rescale, decrypt and
    decode; every stage runs on the device.  Slot values come from host memory and
    the decoded slots go back to it inside the timed region."""
    from fhe_b200 import Engine
    from inputs import codec_values

    eng = Engine(log_coeff_count=14, special_prime_count=1)
    eng.set_stream(stream.cuda_stream)
    eng.set_concurrency(CONCURRENCY)
    eng.seed([5 + rank, 6, 7, 8, 9, 10, 11, 12], [3, 4])
    sk = eng.create_secret_key()
    pk = eng.create_public_key(sk)
    rk = eng.create_relinearization_key(sk)
    B = args.batch
    va = [codec_values(300 + i, eng.slot_count, True) for i in range(B)]
    vb = [codec_values(600 + i, eng.slot_count, True) for i in range(B)]

    def step():
        outs = []
        for a, b in zip(va, vb):
            ca, cb = eng.encrypt(eng.encode(a), pk), eng.encrypt(eng.encode(b), pk)
            prod = eng.rescale(eng.multiply(ca, cb, rk))
            outs.append(eng.decode(eng.decrypt(prod, sk), complex_output=True))
        return outs

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = Engine.kernel_launch_count()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            outs = step()
        stop.record(stream)
        torch.cuda.synchronize()
    launches = Engine.kernel_launch_count() - launches0
    elapsed_max, units = aggregate(start.elapsed_time(stop), float(B * args.steps), world, backend)
    err = max(float(np.max(np.abs(o - a * b))) for o, a, b in zip(outs, va, vb))
    if rank == 0:
        print(json.dumps({
            "metric": "plain CKKS pipeline pairs/s at N=2^14 (encode, encrypt, multiply, "
                      "relinearize, rescale, decrypt, decode)",
            "value": units / (elapsed_max / 1e3), "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64+f64",
            "data": "synthetic (seeded complex slots uniform in [-1, 1], keys made on the device)",
            "config": {"workload": "the reference's default engine (N=2^14, K=1, scale 2^40)",
                       "pairs_per_step": B, "max_error_vs_float64_product": err,
                       "precision_bits": float(-np.log2(err)) if err > 0 else 64.0},
            "cpu_baseline": None,
            "e2e": {"value": units / (elapsed_max / 1e3), "unit": "pairs/s",
                    "h2d_bytes_per_step": int(B * 2 * eng.slot_count * 16),
                    "d2h_bytes_per_step": int(B * eng.slot_count * 16),
                    "note": "slot values from host memory, decoded slots back to it, every "
                            "stage between on the device"},
            "gpu_launches": launches, "clocks": clocks.summary()}), flush=True)
    eng.close()
    return 0


# -------------------------------------------------------------------- main --

def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=16, help="ciphertext pairs per step")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hmult",
                    choices=["hmult", "ntt", "bootstrap", "bootstrap_rotation", "batched",
                             "plain"],
                    help="hmult: the headline; ntt: forward NTT of --batch x 24 limbs at N=2^16; "
                         "bootstrap: --batch ciphertexts bootstrapped per step with a medium "
                         "bootstrap key; bootstrap_rotation: the same with a rotation key; "
                         "batched: --batch uneven HMult+rotate items per step (use 256); "
                         "plain: the N=2^14 pipeline from slot values to decoded slots")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tensor-cores", type=int, default=2, choices=[0, 1, 2],
                    help="base conversions: 0 CUDA cores, 1 INT8 tensor pipe, 2 the engine's "
                         "default (tensor pipe where it measured faster); same words")
    ap.add_argument("--no-bootstrap", action="store_true",
                    help="hmult: leave out the bootstrap measurement of the headline line")
    ap.add_argument("--streams", type=int, default=None,
                    help="worker streams of batch calls (1-8; default: the engine's 4)")
    args = ap.parse_args(argv)
    global CONCURRENCY
    if args.streams is not None:
        CONCURRENCY = args.streams
    rank, world, local = dist_env()

    if args.impl == "reference":
        return run_reference(args, rank)

    import numpy as np
    import torch

    backend = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        backend = "nccl"
    else:
        torch.cuda.set_device(0)

    from fhe_b200 import Engine, NTT_FORM, INCLUDE_SPECIAL, RELINEARIZATION_KEY
    from inputs import uniform_limbs

    # A dedicated stream for the engine and for the timing events (the legacy
    # default stream does not order work on the engine's non-blocking streams).
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    if args.workload == "ntt":
        return run_ntt_microbench(args, torch, np, rank, world, local, backend, stream)
    if args.workload == "plain":
        return run_plain_bench(args, torch, np, rank, world, local, backend, stream)
    if args.workload == "batched":
        return run_batched_bench(args, torch, np, rank, world, local, backend, stream)
    if args.workload in ("bootstrap", "bootstrap_rotation"):
        return run_bootstrap_bench(args, torch, np, rank, world, local, backend, stream)
    eng = Engine(log_coeff_count=LOG_N, special_prime_count=SPECIAL)
    eng.set_stream(stream.cuda_stream)
    eng.set_concurrency(CONCURRENCY)
    n = eng.coeff_count
    level = eng.max_key_switching_level
    mid = eng.moduli_id(level)
    L0 = eng.chains(mid)                      # 28 input limbs
    L = L0 - 1                                # 27 limbs after the lazy rescale
    E = L + SPECIAL
    dnum = (L + SPECIAL - 1) // SPECIAL
    q_in = eng.moduli[mid:mid + L0]
    rng = np.random.default_rng(1234 + rank)
    key = uniform_limbs(rng, eng.moduli[mid:], 2 * eng.partition_count(mid), n)
    rk = eng.upload(key, mid, NTT_FORM | INCLUDE_SPECIAL, RELINEARIZATION_KEY)
    B = args.batch
    # B distinct input pairs (B * 58.7 MB of inputs, larger than the 126 MB L2 for B >= 3)
    pairs = []
    for _ in range(B):
        a = eng.upload(uniform_limbs(rng, q_in, 2, n), mid)
        b = eng.upload(uniform_limbs(rng, q_in, 2, n), mid)
        pairs.append((a, b))

    pa, pb = [p[0] for p in pairs], [p[1] for p in pairs]

    def step():
        # One batch call: the pairs run concurrently on the engine's worker streams.
        outs = eng.multiply_relinearize_rescale_batch(pa, pb, rk)
        for o in outs:
            o.free()

    def per_call_step():
        outs = [eng.multiply_relinearize_rescale(a, b, rk) for a, b in pairs]
        for o in outs:
            o.free()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if backend:
        torch.distributed.barrier()
    launches0 = Engine.kernel_launch_count()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            step()
        stop.record(stream)
        torch.cuda.synchronize()
    launches = Engine.kernel_launch_count() - launches0
    elapsed = start.elapsed_time(stop)
    if backend:
        torch.distributed.barrier()
    elapsed_max, units = aggregate(elapsed, float(B * args.steps), world, backend)
    value = units / (elapsed_max / 1e3)

    def timed_steps(fn, profile: bool):
        """Device ms of args.steps calls of fn; with profile, per-family event times
        too (one stream, so each kernel's time is its own)."""
        fn()
        torch.cuda.synchronize()
        if profile:
            eng.set_concurrency(1)
            eng.profile_reset()
            eng.set_profiling(True)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(args.steps):
            fn()
        s1.record(stream)
        torch.cuda.synchronize()
        p = None
        if profile:
            eng.set_profiling(False)
            eng.set_concurrency(CONCURRENCY)
            p = eng.profile()
        ms, u = aggregate(s0.elapsed_time(s1), float(B * args.steps), world, backend)
        return u / (ms / 1e3), p

    # The same pairs one call each (no batch), and the per-kernel profile.
    per_call_value, _ = timed_steps(per_call_step, False)
    _, prof = timed_steps(step, True)

    # ---- roofline of the dominant kernel family (event-timed in the region above)
    bytes_per = kernel_bytes(L, E, dnum, n)
    dominant = max(prof, key=lambda k: prof[k][1]) if prof else None
    peak, peak_kind = measured_peaks()
    roofline = None
    if dominant:
        cnt, ms = prof[dominant]
        avg_ms = ms / cnt
        achieved = bytes_per.get(dominant, 0) / (avg_ms / 1e3) / 1e9
        traffic = None
        tpath = os.path.join(HERE, "profiles", "traffic.json")
        if os.path.exists(tpath):
            traffic = json.load(open(tpath)).get(dominant)
        integer, tensor = pipe_figures(prof, args.steps, B, n, L, SPECIAL, clocks.summary()["sm_mhz"],
                                       torch.cuda.get_device_properties(0).multi_processor_count)
        roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak,
                    "limiter": "integer instruction issue: every transform and Montgomery product "
                               "is 64-bit integer arithmetic on the CUDA cores (integer_pipe); the "
                               "HBM fraction and the INT8 tensor-pipe fraction (tensor_pipe) are "
                               "both small",
                    "integer_pipe": integer, "tensor_pipe": tensor,
                    "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                    "peak_source": peak_kind, "avg_launch_ms": avg_ms,
                    "algorithmic_bytes_per_launch": bytes_per.get(dominant),
                    # of the kernel time of one stream (the profiled pass runs the
                    # batch on one stream, as ncu's serialised launch list does)
                    "share_of_kernel_time": ms / sum(v[1] for v in prof.values()),
                    "kernel_ms_per_step": {k: v[1] / args.steps for k, v in prof.items()}}

    # ---- the same step with the base conversions on the CUDA cores (OFF), on the
    # tensor pipe (AUTO, the default at 10 special primes) and with ModUp's and
    # ModDown's NTTs on the tensor pipe as well (ON); every form gives the same words.
    def timed_form(mode: int):
        eng.set_tensor_cores(mode)
        form_value, _ = timed_steps(step, False)
        _, p = timed_steps(step, True)
        eng.set_tensor_cores(2)
        fam = "mod_down_epilogue_tc" if "mod_down_epilogue_tc" in p else "mod_down_epilogue"
        cnt, fam_ms = p.get(fam, (0, 0.0))
        up = "mod_up_ntt_tc" if "mod_up_ntt_tc" in p else "mod_up_ntt"
        up_cnt, up_ms = p.get(up, (0, 0.0))
        if up == "mod_up_ntt_tc":  # the tensor-pipe contraction and the NTT that follows it
            up_ms += p.get("mod_up_contract_tc", (0, 0.0))[1]
        down = "mod_down_intt_tc" if "mod_down_intt_tc" in p else "mod_down_intt"
        return {"value": form_value, "unit": "ct/s", "mode": ["off", "on", "auto"][mode],
                "mod_down_kernel": fam,
                "mod_down_avg_launch_ms": fam_ms / cnt if cnt else None,
                "mod_down_ms_per_step": fam_ms / args.steps,
                "mod_up_family": up, "mod_up_avg_launch_ms": up_ms / up_cnt if up_cnt else None,
                "mod_up_ms_per_step": up_ms / args.steps,
                "mod_down_ntt_family": down, "mod_down_ntt_ms_per_step": p.get(down, (0, 0.0))[1] / args.steps}

    forms = {"tensor_core": timed_form(2), "tensor_core_with_ntt": timed_form(1),
             "cuda_core": timed_form(0)}

    # ---- end to end through the C ABI with pinned host buffers
    in_words = 2 * L0 * n
    out_words = 2 * (L - 1) * n
    pin_in = torch.empty((B, 2, in_words), dtype=torch.int64, pin_memory=True)
    pin_out = torch.empty((B, out_words), dtype=torch.int64, pin_memory=True)
    for i in range(B):
        pin_in[i, 0].copy_(torch.from_numpy(uniform_limbs(rng, q_in, 2, n).reshape(-1)))
        pin_in[i, 1].copy_(torch.from_numpy(uniform_limbs(rng, q_in, 2, n).reshape(-1)))

    def e2e_step():
        # Batch calls of CONCURRENCY pairs: a chunk's kernels start once its own
        # uploads land, so copies and kernels of neighbouring chunks overlap.
        for c0 in range(0, B, CONCURRENCY):
            idx = range(c0, min(B, c0 + CONCURRENCY))
            ins_a = [eng.upload_from_pointer(pin_in[i, 0].data_ptr(), mid, 2) for i in idx]
            ins_b = [eng.upload_from_pointer(pin_in[i, 1].data_ptr(), mid, 2) for i in idx]
            outs = eng.multiply_relinearize_rescale_batch(ins_a, ins_b, rk)
            for i, o in zip(idx, outs):
                eng.download_to_pointer(o, pin_out[i].data_ptr(), wait=False)
            # No wait: every object is freed behind the work that reads it.
            for d in ins_a + ins_b + outs:
                d.free()

    for _ in range(args.warmup):  # the stream-ordered pool reaches its steady size
        e2e_step()
    eng.synchronize()
    torch.cuda.synchronize()
    if backend:
        torch.distributed.barrier()
    e_steps = args.steps
    s2, t2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(e_steps):
        e2e_step()
    eng.synchronize()  # the last results are in host memory
    t2.record(stream)
    torch.cuda.synchronize()
    e_elapsed, e_units = aggregate(s2.elapsed_time(t2), float(B * e_steps), world, backend)
    e2e_value = e_units / (e_elapsed / 1e3)

    # ---- the host link alone: the step's input bytes from the same pinned buffer to
    # the device in one copy, the ceiling of the end-to-end rate
    dev_in = torch.empty(pin_in.shape, dtype=torch.int64, device="cuda")
    dev_in.copy_(pin_in, non_blocking=True)
    torch.cuda.synchronize()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for _ in range(3):
        dev_in.copy_(pin_in, non_blocking=True)
    h1.record(stream)
    torch.cuda.synchronize()
    h2d_bytes = B * 2 * in_words * 8
    h2d_gbs = 3 * h2d_bytes / (h0.elapsed_time(h1) / 1e3) / 1e9
    # Both directions at once, as the end-to-end step moves them: the step's inputs
    # to the device and its results back, on two streams.
    dev_out = torch.empty(pin_out.shape, dtype=torch.int64, device="cuda")
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d0.record(stream)
    up.wait_event(d0)
    down.wait_event(d0)
    for _ in range(3):
        with torch.cuda.stream(up):
            dev_in.copy_(pin_in, non_blocking=True)
        with torch.cuda.stream(down):
            pin_out.copy_(dev_out, non_blocking=True)
    stream.wait_stream(up)
    stream.wait_stream(down)
    d1.record(stream)
    torch.cuda.synchronize()
    duplex_ms = d0.elapsed_time(d1) / 3
    del dev_in, dev_out

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline_sample()
        line = {
            "metric": METRIC, "value": value, "unit": "ct/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded uniform residues, random relinearization key)",
            "config": {"workload": WORKLOAD, "pairs_per_step": B, "log_n": LOG_N,
                       "api": "fhe_multiply_relinearize_rescale_batch", "streams": CONCURRENCY,
                       "per_call_ct_s": per_call_value,
                       "special_prime_count": SPECIAL, "input_limbs": L0,
                       "relinearize_limbs": L, "dnum": dnum, "parallelism": f"replicas{world}",
                       "l2": f"inputs larger than L2 ({B} pairs x {2 * 2 * L0 * n * 8 / 1e6:.1f} MB)"},
            "roofline": roofline,
            "bconv_forms": forms,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "ct/s",
                    "h2d_bytes_per_step": B * 2 * in_words * 8,
                    "d2h_bytes_per_step": B * out_words * 8,
                    "h2d_gbs_measured": h2d_gbs,
                    "h2d_ceiling_ct_s": B / (h2d_bytes / (h2d_gbs * 1e9)),
                    "duplex_copy_ms_per_step": duplex_ms,
                    "duplex_ceiling_ct_s": B / (duplex_ms / 1e3)},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
    del pairs, pa, pb, rk
    eng.close()
    # The other half of the headline metric: bootstrap ms (medium bootstrap key, 8
    # ciphertexts per step), measured in the same run under its own clock record.
    boot = None
    if not args.no_bootstrap:
        boot = bootstrap_measure(args, torch, np, rank, world, local, backend, stream, True,
                                 BOOTSTRAP_BATCH)
    if rank == 0:
        line["bootstrap"] = boot
        print(json.dumps(line), flush=True)
    if backend:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
