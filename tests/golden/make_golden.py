"""Regenerate the golden fixtures under tests/golden/.

1. ``ntt_kat.json`` and ``precomputed_kat.json``: the known-answer vectors of the
   reference's own unit tests (test/operation/ntt.cpp and
   test/ckks/precomputed/default.cpp), read as text.
2. ``ref_ops.json``: outputs of the compiled reference library (oracle/_ref, built
   by ``make -C oracle ref``) on seeded inputs (tests/golden/inputs.py): NTT /
   iNTT, tensor, relinearize, rescale and engine multiply+relinearize+rescale,
   stored as SHA-256 digests of the int64 limbs (full arrays for N <= 16).

Needs the reference tree ($FHE_REFERENCE, else the ``reference`` directory beside
the repository); the tests read only the committed JSON.  Usage:
``python tests/golden/make_golden.py`` (every fixture) or
``python tests/golden/make_golden.py --headline`` (ref_ops_c10.json only: the
reference_ops digests at N = 2^16 with 10 special primes).
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from inputs import ROTATION_KEY_DELTAS, arith_inputs, codec_values, digest_doubles, digest_list, key_switch_inputs, TIERS, case_inputs, digest  # noqa: E402

REF = os.environ.get("FHE_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))


def _tests(text: str):
    """Split a googletest file into {name: body}."""
    out = {}
    for m in re.finditer(r"TEST\((\w+),\s*(\w+)\)\s*\{", text):
        start = m.end()
        depth, i = 1, start
        while depth:
            depth += {"{": 1, "}": -1}.get(text[i], 0)
            i += 1
        out[f"{m.group(1)}.{m.group(2)}"] = text[start:i - 1]
    return out


def _ints(body: str):
    return [int(eval(v.strip())) for v in body.replace("\n", " ").split(",") if v.strip()]


def parse_ntt_kats():
    text = open(os.path.join(REF, "test/operation/ntt.cpp")).read()
    kats = []
    for name, body in _tests(text).items():
        if not re.match(r"^NTT\.I?NTT(Inplace)?\d$", name):
            continue  # split/unit helpers and composite tests are not single transforms
        call = re.search(r"desilo::fhe::(ntt|intt)\((\w+),\s*(\w+),\s*(\w+)", body)
        if not call:
            continue
        kind, src, dst, table = call.groups()
        arrays = {m.group(1): _ints(m.group(2))
                  for m in re.finditer(r"int64_t\s+(\w+)\[\d*\]\s*\{([^}]*)\}", body)}
        scalars = {m.group(1): int(m.group(2))
                   for m in re.finditer(r"(?:uint64_t|int64_t|int)\s+(\w+)\s*=\s*(\d+)\s*;", body)}
        kats.append(dict(name=name, kind=kind, x=arrays[src], table=arrays[table],
                         q=scalars["q"], k=scalars["k"], expected=arrays["expected"]))
    return kats


def parse_random_kats():
    """test/random/random.cpp: ChaCha20 blocks and the rand_int / discrete_gaussian
    outputs for the test state (seed words 1..8, nonce 9, 10, counter 0), plus the
    sampler's CDT tree literal from src/random/gaussian_sampler.cpp."""
    text = open(os.path.join(REF, "test/random/random.cpp")).read()
    blocks = re.search(r"expected_chacha20\[4\]\[16\]\{(.*?)\};", text, re.S).group(1)
    chacha = [_ints(b) for b in re.findall(r"\{([^{}]*)\}", blocks)]
    arrays = {m.group(1): _ints(m.group(2))
              for m in re.finditer(r"int64_t\s+(expected_\w+)\[\d+\]\{([^}]*)\}", text)}
    sampler = open(os.path.join(REF, "src/random/gaussian_sampler.cpp")).read()
    tree = re.search(r"tree_128_3_2\[\d+\]\{(.*?)\};", sampler, re.S).group(1)
    tree_words = [int(v.strip().rstrip("u")) for v in tree.replace("\n", " ").split(",") if v.strip()]
    return dict(seed=[1, 2, 3, 4, 5, 6, 7, 8], nonce=[9, 10], chacha20=chacha,
                rand_int_10=arrays["expected_rand_int"],
                rand_int_10_shift_10=arrays["expected_rand_int_shifted"],
                discrete_gaussian=arrays["expected_discrete_gaussian"], cdt_tree=tree_words)


def parse_precomputed_kats():
    text = open(os.path.join(REF, "test/ckks/precomputed/default.cpp")).read()
    out = {}
    for name, body in _tests(text).items():
        tier = re.search(r'from_tier\("(\w+)"\)', body)
        if tier:
            tier = tier.group(1)
        elif "for_bootstrap()" in body:
            tier = "bootstrap_gold"
        else:
            continue
        vectors = {}
        for m in re.finditer(r"std::vector<(u?int64_t)>\s+(\w+)\s*=\s*\{(.*?)\};", body, re.S):
            vectors[m.group(2)] = _ints(m.group(3))
        for m in re.finditer(r"std::vector<std::vector<int64_t>>\s+(\w+)\s*=\s*\{(.*?)\};", body, re.S):
            rows = re.findall(r"\{([^{}]*)\}", m.group(2))
            vectors[m.group(1)] = [_ints(r) for r in rows]
        out[name] = dict(tier=tier, vectors=vectors)
    return out


def key_switch_ops(e, seed, q, n, mid, K, a, rk):
    """Rotation, conjugation, key switch, level down and mixed-level multiply
    through the reference's engine (and core, for switch_key)."""
    x = key_switch_inputs(seed, q, n, mid, K)
    kmid = x["key_moduli_id"]
    res = {}
    fks = [e.fixed_rotation_key(k, kmid, d) for k, d in zip(x["rotation_keys"], ROTATION_KEY_DELTAS)]
    ck = e.conjugation_key(x["conjugation_key"], kmid)
    scale = 2.0 ** 40
    level = e.chains(mid) - 2
    res["rotate_1"] = e.rotate(e.text(a, mid, flag=0, scale=scale), fks[0]).limbs()
    res["rotate_4_ntt"] = e.rotate(e.text(a, mid, flag=2, scale=scale), fks[2]).limbs()
    res["rotate_keys_7"] = e.rotate_keys(e.text(a, mid, flag=0, scale=scale), fks, 7).limbs()
    res["conjugate"] = e.conjugate(e.text(a, mid, flag=0, scale=scale), ck).limbs()
    res["switch_key"] = e.core_switch_key(e.text(a, mid, flag=0),
                                          e.switching_key(x["switching_key"], mid)).limbs()
    res["rotate_plain_3"] = e.rotate_plain(e.text(a[:1], mid, flag=0, kind=5), 3).limbs()
    res["rotate_plain_3_ntt"] = e.rotate_plain(e.text(a[:1], mid, flag=2, kind=5), 3).limbs()
    res["conjugate_plain"] = e.conjugate(e.text(a[:1], mid, flag=0, kind=5)).limbs()
    res["conjugate_plain_ntt"] = e.conjugate(e.text(a[:1], mid, flag=2, kind=5)).limbs()
    if level >= 1:
        res["level_down"] = e.level_down(e.text(a, mid, flag=0, scale=scale), level - 1).limbs()
        res["level_down_ntt"] = e.level_down(e.text(a, mid, flag=2, scale=scale), 0).limbs()
    if level >= 1 and mid >= 1:  # a rescaled text never sits at moduli id 0
        res["level_down_rescaled"] = e.level_down(e.text(a, mid, flag=4, scale=scale),
                                                  level).limbs()
    try:
        m = e.multiply(e.text(a, mid, flag=0, scale=scale), e.text(x["b_next"], mid + 1, flag=0,
                                                                   scale=scale), rk)
        res["multiply_mixed_levels"] = m.limbs()
    except RuntimeError:
        pass
    return res


REFERENCE_OPS_PLAN = [("pebble", [0, 1, 5]), ("sand", [2]), ("iron", [1]), ("bronze", [1, 3]),
                      ("silver", [1]), ("gold", [5]), ("bootstrap_gold", [1])]
# The headline key-switching configuration: N = 2^16 with 10 special primes.  Moduli
# id 1 is the key-switching level (28 limbs, partitions [8, 10, 10]); id 2 has a
# 7-limb first partition; id 5 has 24 limbs and partitions [4, 10, 10].
HEADLINE_OPS_PLAN = [("c10", [1, 2, 5])]


def reference_ops(plan=REFERENCE_OPS_PLAN, seed=1000, threads=1):
    from oracle import ref

    cases = []
    for tier, moduli_ids in plan:
        log_n, K, preset = TIERS[tier]
        e = ref.Engine(log_n=log_n, special_prime_count=K, preset=preset, threads=threads)
        q = e.tables()["q"]
        n = e.n
        for mid in moduli_ids:
            seed += 1
            a, b, ct3, key = case_inputs(seed, q, n, mid, K)
            res = {}
            x = e.text(a, mid, flag=0)
            xn = e.core_to_ntt(x)
            res["to_ntt"] = xn.limbs()
            res["to_intt"] = e.core_to_intt(e.text(a, mid, flag=2)).limbs()
            res["tensor"] = e.core_tensor(e.text(a, mid, flag=2), e.text(b, mid, flag=2)).limbs()
            rk = e.relin_key(key, mid)
            res["relinearize"] = e.core_relinearize(e.text(ct3, mid, flag=2), rk).limbs()
            res["rescale"] = e.core_rescale(e.text(a, mid, flag=0)).limbs()
            try:
                m = e.multiply(e.text(a, mid, flag=0), e.text(b, mid, flag=0), rk)
                res["mult_relin_rescale"] = e.rescale(m).limbs()
            except RuntimeError:
                pass
            arrays = {k: v.tolist() for k, v in res.items()} if n <= 16 else None
            res.update(key_switch_ops(e, seed, q, n, mid, K, a, rk))
            entry = dict(tier=tier, log_n=log_n, special_prime_count=K, preset=preset,
                         moduli_id=mid, seed=seed, moduli=[int(v) for v in q],
                         digests={k: digest(v) for k, v in res.items()})
            if arrays is not None:
                entry["arrays"] = arrays
            cases.append(entry)
    return cases


# (tier, log_slot_count): full slots, plus one sparse-slot engine.
CODEC_PLAN = [("pebble", -1), ("bronze", -1), ("bronze", 10), ("bootstrap_gold", -1)]


def codec_cases():
    """Encode / decode through the reference's engine (encode_unit, decode_unit,
    decode_complex_unit_plaintext) on seeded slot values."""
    from oracle import ref

    cases = []
    seed = 5000
    for tier, log_slot in CODEC_PLAN:
        log_n, K, preset = TIERS[tier]
        e = ref.Engine(log_n=log_n, special_prime_count=K, preset=preset, log_slot=log_slot)
        full = e.chain_count - 2
        for level in sorted({full, full - 1, 1}):
            for kind in ("real", "complex"):
                seed += 1
                vals = codec_values(seed, e.slot_count, kind == "complex")
                pt = e.encode(vals, level, real=kind == "real")
                # digest before decoding: the reference's decode reduces the limbs of
                # its input in place (make_unsigned_reduce_2q_to_q, core_decode.cpp:82)
                encoded = digest(pt.limbs())
                dec = e.decode_real(pt) if kind == "real" else e.decode(pt)
                info = pt.info()
                cases.append(dict(tier=tier, log_n=log_n, special_prime_count=K, preset=preset,
                                  log_slot=log_slot, level=level, kind=kind, seed=seed,
                                  moduli_id=info["moduli_id"], scale_bits=e.scale_bits,
                                  moduli=[int(v) for v in e.tables()["q"]],
                                  encode=encoded, decode=digest_doubles(dec),
                                  max_error=float(np.max(np.abs(dec - vals)))))
    return cases


KEYGEN_TIERS = ["pebble", "iron", "bronze", "silver", "bootstrap_gold"]
KEYGEN_SEED = (11, 22, 33, 44, 55, 66, 77, 88)
KEYGEN_NONCE = (5, 9)


def keygen_cases():
    """Keys, encryptions and decryptions through the reference's engine after
    reseeding its ChaCha20 stream; the calls run in this order, so each output
    depends on the stream position the previous calls left."""
    from oracle import ref

    cases = []
    for tier in KEYGEN_TIERS:
        log_n, K, preset = TIERS[tier]
        e = ref.Engine(log_n=log_n, special_prime_count=K, preset=preset)
        e.seed(KEYGEN_SEED, KEYGEN_NONCE)
        out = {}
        sk = e.create_secret_key()
        out["secret_key"] = sk.limbs()
        pk = e.create_public_key(sk)
        out["public_key"] = pk.limbs()
        rk = e.create_relinearization_key(sk)
        out["relinearization_key"] = rk.limbs()
        fk = e.create_fixed_rotation_key(sk, 3)
        out["fixed_rotation_key_3"] = fk.limbs()
        ck = e.create_conjugation_key(sk)
        out["conjugation_key"] = ck.limbs()
        vals = codec_values(7000 + log_n, e.slot_count, True)
        level = e.max_level
        pt = e.encode(vals, level)
        out["plaintext"] = pt.limbs()
        ct_pk = e.encrypt(pt, pk)
        out["encrypt_public"] = ct_pk.limbs()
        ct_sk = e.encrypt(pt, sk)
        out["encrypt_secret"] = ct_sk.limbs()
        dec = e.decrypt(ct_pk, sk)
        out["decrypt_public"] = dec.limbs()
        slots = e.decode(dec)
        cases.append(dict(tier=tier, log_n=log_n, special_prime_count=K, preset=preset,
                          seed=list(KEYGEN_SEED), nonce=list(KEYGEN_NONCE), values_seed=7000 + log_n,
                          level=level, moduli=[int(v) for v in e.tables()["q"]],
                          digests={k: digest(v) for k, v in out.items()},
                          decoded=digest_doubles(slots),
                          max_error=float(np.max(np.abs(slots - vals)))))
    return cases


ARITH_PLAN = [("pebble", 2), ("bronze", 1), ("silver", 2), ("bootstrap_gold", 3)]


def arith_cases():
    """Ciphertext arithmetic through the reference's engine on uniform operands.
    Each case lists (op, operand names, flags); flags: 2 NTT form, 4 rescaled.  Every
    call gets fresh input objects: the reference reduces some NTT-form inputs in place."""
    from oracle import ref

    plan = [
        ("add", "a:0", "b:0"), ("add", "a:2", "low:2"), ("add", "trio:2", "a:2"),
        ("add", "a:4", "b:0"), ("subtract", "a:0", "b:0"), ("subtract", "a:2", "trio:2"),
        ("subtract", "trio:0", "low:0"), ("add_plain", "a:0", "plain:0"),
        ("add_plain", "a:2", "plain:0"), ("subtract_plain", "a:2", "plain:0"),
        ("subtract_from_plain", "a:2", "plain:0"), ("subtract_from_plain", "a:0", "plain:0"),
        ("multiply_plain", "a:0", "plain:0"), ("multiply_plain", "a:2", "plain:2"),
        ("negate", "a:2"), ("negate", "trio:0"), ("square", "a:0"), ("square_relinearize", "a:2"),
        ("add_scalar", "a:0", 0.37), ("add_scalar", "a:2", -1.25), ("subtract_scalar", "b:0", 2.5),
        ("multiply_scalar", "a:0", 0.71), ("multiply_scalar", "b:2", -2.5),
        ("multiply_integer", "a:2", -3),
    ]
    cases = []
    seed = 9000
    for tier, mid in ARITH_PLAN:
        log_n, K, preset = TIERS[tier]
        e = ref.Engine(log_n=log_n, special_prime_count=K, preset=preset)
        q = e.tables()["q"]
        seed += 1
        x = arith_inputs(seed, q, e.n, mid, K)
        level = e.chains(mid) - 2
        probe = e.encode(np.zeros(e.slot_count), level)
        scale = probe.info()["scale"]
        low_scale = e.encode(np.zeros(e.slot_count), level - 1).info()["scale"]

        def text(spec):
            name, flag = spec.split(":")
            flag = int(flag)
            m = mid + 1 if name == "low" else mid
            kind = 5 if name == "plain" else 4
            s = low_scale if name == "low" else scale
            return e.text(x[name], m, flag=flag, kind=kind, scale=s)

        rk = e.relin_key(x["key"], mid)
        digests = {}
        for step in plan:
            op = step[0]
            key = "|".join(str(v) for v in step)
            if op in ref.Engine.SCALAR:
                out = e.scalar(op, text(step[1]), step[2])
            elif op == "square_relinearize":
                out = e.arith(op, text(step[1]), rk)
            elif len(step) == 2:
                out = e.arith(op, text(step[1]))
            else:
                out = e.arith(op, text(step[1]), text(step[2]))
            digests[key] = digest(out.limbs())
        cases.append(dict(tier=tier, log_n=log_n, special_prime_count=K, preset=preset,
                          moduli_id=mid, seed=seed, scale=scale, low_scale=low_scale,
                          moduli=[int(v) for v in q], digests=digests))
    return cases


BOOTSTRAP_SEED = (101, 202, 303, 404, 505, 606, 707, 808)
BOOTSTRAP_NONCE = (7, 3)


def bootstrap_cases():
    """Bootstrapping through the reference's engine (bootstrap preset, N = 2^16,
    4 special primes, 3 stages) after reseeding: secret, relinearization, conjugation,
    rotation and small bootstrap keys, a secret-key encryption at level 3, then
    bootstrap(ct, rk, ck, rotation key, small bootstrap key, 3)."""
    from oracle import ref

    log_n, K, preset = TIERS["bootstrap_gold"]
    e = ref.Engine(log_n=log_n, special_prime_count=K, preset=preset, threads=os.cpu_count())
    e.seed(BOOTSTRAP_SEED, BOOTSTRAP_NONCE)
    out = {}
    sk = e.create_secret_key()
    out["secret_key"] = sk.limbs()
    rk = e.create_relinearization_key(sk)
    out["relinearization_key"] = rk.limbs()
    ck = e.create_conjugation_key(sk)
    out["conjugation_key"] = ck.limbs()
    rotk, views = e.create_rotation_key(sk)
    out["rotation_key_1"] = views[0][0].limbs()
    rotation_keys = [digest(v.limbs()) for v, _ in views]
    sbk, (to_sparse, to_dense) = e.create_small_bootstrap_key(sk)
    out["to_sparse"] = to_sparse.limbs()
    out["to_dense"] = to_dense.limbs()
    vals = codec_values(4242, e.slot_count, True)
    pt = e.encode(vals, 3)
    ct = e.encrypt(pt, sk)
    out["ciphertext"] = ct.limbs()
    boot = e.bootstrap(ct, rk, ck, rotk, sbk, 3)
    out["bootstrapped"] = boot.limbs()
    info = boot.info()
    dec = e.decode(e.decrypt(boot, sk))
    return [dict(tier="bootstrap_gold", log_n=log_n, special_prime_count=K, preset=preset,
                 seed=list(BOOTSTRAP_SEED), nonce=list(BOOTSTRAP_NONCE), values_seed=4242,
                 encrypt_level=3, stage_count=3, moduli=[int(v) for v in e.tables()["q"]],
                 rotation_deltas=[d for _, d in views], rotation_keys=rotation_keys,
                 output_moduli_id=info["moduli_id"],
                 output_level=info["level"], digests={k: digest(v) for k, v in out.items()},
                 decoded=digest_doubles(dec), max_error=float(np.max(np.abs(dec - vals))))]


def bootstrap_key_cases():
    """Bootstrapping with a bootstrap key (bootstrap preset, N = 2^16, K = 4, 3 stages,
    "medium"): after reseeding, secret, relinearization and conjugation keys, then
    create_bootstrap_key (every fixed rotation key, the stages' diagonals, the small
    bootstrap key), a secret-key encryption at level 3 and bootstrap(ct, rk, ck, bk)."""
    from oracle import ref

    log_n, K, preset = TIERS["bootstrap_gold"]
    e = ref.Engine(log_n=log_n, special_prime_count=K, preset=preset, threads=os.cpu_count())
    e.seed(BOOTSTRAP_SEED, BOOTSTRAP_NONCE)
    out = {}
    sk = e.create_secret_key()
    out["secret_key"] = sk.limbs()
    rk = e.create_relinearization_key(sk)
    out["relinearization_key"] = rk.limbs()
    ck = e.create_conjugation_key(sk)
    out["conjugation_key"] = ck.limbs()
    bk = e.create_bootstrap_key(sk, 3, "medium")
    keys = e.bootstrap_key_rotation_keys(bk)
    rotation_keys = [[d, digest(k.limbs())] for k, d in keys]
    stages = []
    for to_slot in (1, 0):
        for stage in range(3):
            level, inner, outer, _ = e.bootstrap_key_stage(bk, to_slot, stage)
            diagonals = []
            for o in range(outer):
                for i in range(inner):
                    d = e.bootstrap_key_diagonal(bk, to_slot, stage, o, i)
                    if d is not None:
                        diagonals.append(digest(d.limbs()))
            stages.append(dict(to_slot=to_slot, stage=stage, level=level, inner=inner,
                               outer=outer, diagonal_count=len(diagonals),
                               diagonals=digest_list(diagonals)))
    to_sparse, to_dense = e.bootstrap_key_small(bk)
    out["to_sparse"] = to_sparse.limbs()
    out["to_dense"] = to_dense.limbs()
    vals = codec_values(4242, e.slot_count, True)
    ct = e.encrypt(e.encode(vals, 3), sk)
    out["ciphertext"] = ct.limbs()
    boot = e.bootstrap_with_key(ct, rk, ck, bk)
    out["bootstrapped"] = boot.limbs()
    info = boot.info()
    dec = e.decode(e.decrypt(boot, sk))
    return [dict(tier="bootstrap_key_gold", log_n=log_n, special_prime_count=K, preset=preset,
                 seed=list(BOOTSTRAP_SEED), nonce=list(BOOTSTRAP_NONCE), values_seed=4242,
                 encrypt_level=3, stage_count=3, size="medium",
                 moduli=[int(v) for v in e.tables()["q"]], rotation_keys=rotation_keys,
                 stages=stages, output_moduli_id=info["moduli_id"], output_level=info["level"],
                 digests={k: digest(v) for k, v in out.items()}, decoded=digest_doubles(dec),
                 max_error=float(np.max(np.abs(dec - vals))))]


PIPELINE_SEED = (31, 41, 59, 26, 53, 58, 97, 93)
PIPELINE_NONCE = (2, 7)


def pipeline_cases():
    """The plain CKKS pipeline of the reference's default engine (N = 2^14, one
    special prime) and of the gold tier: after reseeding, secret, public and
    relinearization keys; two complex vectors encoded at the top level and encrypted
    with the public key; multiply with the relinearization key, rescale, decrypt,
    decode.  Words of every ciphertext and the decoded slots, and the error against
    the float64 product."""
    from oracle import ref

    cases = []
    for tier in ("bronze", "gold"):
        log_n, K, preset = TIERS[tier]
        e = ref.Engine(log_n=log_n, special_prime_count=K, preset=preset, threads=os.cpu_count())
        e.seed(PIPELINE_SEED, PIPELINE_NONCE)
        out = {}
        sk = e.create_secret_key()
        pk = e.create_public_key(sk)
        rk = e.create_relinearization_key(sk)
        out["public_key"] = pk.limbs()
        va = codec_values(11, e.slot_count, True)
        vb = codec_values(12, e.slot_count, True)
        a = e.encrypt(e.encode(va), pk)
        b = e.encrypt(e.encode(vb), pk)
        out["ct_a"], out["ct_b"] = a.limbs(), b.limbs()
        product = e.multiply(a, b, rk)
        out["product"] = product.limbs()
        rescaled = e.rescale(product)
        out["rescaled"] = rescaled.limbs()
        info = rescaled.info()
        slots = e.decode(e.decrypt(rescaled, sk))
        cases.append(dict(tier=tier, log_n=log_n, special_prime_count=K, preset=preset,
                          seed=list(PIPELINE_SEED), nonce=list(PIPELINE_NONCE), values_seeds=[11, 12],
                          moduli=[int(v) for v in e.tables()["q"]],
                          rescaled_moduli_id=info["moduli_id"], rescaled_level=info["level"],
                          digests={k: digest(v) for k, v in out.items()},
                          decoded=digest_doubles(slots),
                          max_error=float(np.max(np.abs(slots - va * vb)))))
    return cases


def headline_ops():
    """ref_ops_c10.json: the reference_ops digests at N = 2^16 with 10 special primes
    (the benchmarked parameter set), on the reference's worker pool."""
    return reference_ops(HEADLINE_OPS_PLAN, seed=3000, threads=os.cpu_count())


def main():
    if sys.argv[1:] == ["--headline"]:
        cases = headline_ops()
        with open(os.path.join(HERE, "ref_ops_c10.json"), "w") as f:
            json.dump(cases, f, indent=1)
        return
    with open(os.path.join(HERE, "ntt_kat.json"), "w") as f:
        json.dump(parse_ntt_kats(), f, indent=1)
    with open(os.path.join(HERE, "precomputed_kat.json"), "w") as f:
        json.dump(parse_precomputed_kats(), f, indent=1)
    with open(os.path.join(HERE, "random_kat.json"), "w") as f:
        json.dump(parse_random_kats(), f, indent=1)
    cases = reference_ops()  # computed before the file is opened: a failure keeps the old one
    with open(os.path.join(HERE, "ref_ops.json"), "w") as f:
        json.dump(cases, f, indent=1)
    codec = codec_cases()
    with open(os.path.join(HERE, "codec.json"), "w") as f:
        json.dump(codec, f, indent=1)
    arith = arith_cases()
    with open(os.path.join(HERE, "arith.json"), "w") as f:
        json.dump(arith, f, indent=1)
    boot = bootstrap_cases()
    with open(os.path.join(HERE, "bootstrap.json"), "w") as f:
        json.dump(boot, f, indent=1)
    boot_key = bootstrap_key_cases()
    with open(os.path.join(HERE, "bootstrap_key.json"), "w") as f:
        json.dump(boot_key, f, indent=1)
    pipeline = pipeline_cases()
    with open(os.path.join(HERE, "pipeline.json"), "w") as f:
        json.dump(pipeline, f, indent=1)
    keygen = keygen_cases()
    with open(os.path.join(HERE, "keygen.json"), "w") as f:
        json.dump(keygen, f, indent=1)


if __name__ == "__main__":
    main()
