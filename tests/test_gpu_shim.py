"""The reference's own programs on the B200 engine: examples/encrypt_decrypt.cpp,
examples/multiply_vector.cpp and shim/engine_check.cpp are each built twice by
shim/Makefile, against the reference's CPU engine and, through GpuCKKSEngine
(shim/gpu_ckks_engine.cpp, the reference's AbstractEngine over the C ABI), against
the B200 engine.  Both builds draw fresh keys from the system random device, so
their outputs agree to within the CKKS noise, not word for word: every printed
slot must match within 1e-6, and every error against the plaintext computation
must stay below 1e-6."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BUILD = os.path.join(ROOT, "shim", "_build")


def _run(name):
    path = os.path.join(BUILD, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built (make -C shim needs the reference tree)")
    out = subprocess.run([path], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    return out.stdout


def _numbers(text):
    return [float(v) for v in re.findall(r"[-+]?\d+\.?\d*(?:e[-+]?\d+)?", text)]


@pytest.mark.parametrize("example", ["encrypt_decrypt", "multiply_vector"])
def test_reference_example_runs_unchanged_on_the_gpu(example):
    cpu, gpu = _run(f"{example}_cpu"), _run(f"{example}_gpu")
    cpu_lines, gpu_lines = cpu.strip().splitlines(), gpu.strip().splitlines()
    labels = [l.strip() for l in gpu_lines if l.rstrip().endswith(":")]
    assert labels == [l.strip() for l in cpu_lines if l.rstrip().endswith(":")]
    assert labels == ["message:", "decrypted:"]
    message = _numbers(gpu_lines[1])
    decrypted = _numbers(gpu_lines[3])
    assert message == _numbers(cpu_lines[1])
    want = message if example == "encrypt_decrypt" else [m * m for m in message]
    assert len(decrypted) == len(want) == 10
    for g, c, w in zip(decrypted, _numbers(cpu_lines[3]), want):
        assert abs(g - w) < 1e-6 and abs(g - c) < 1e-6


def test_engine_interface_walk_matches_the_cpu_engine():
    cpu, gpu = _run("engine_check_cpu"), _run("engine_check_gpu")
    cpu_rows = dict(l.split(" err ", 1) for l in cpu.strip().splitlines())
    gpu_rows = dict(l.split(" err ", 1) for l in gpu.strip().splitlines())
    assert list(gpu_rows) == list(cpu_rows) and len(gpu_rows) >= 15
    for name, row in gpu_rows.items():
        err, values = row.split(":")
        assert float(err) < 1e-6, (name, err)
        for g, c in zip(_numbers(values), _numbers(cpu_rows[name].split(":")[1])):
            assert abs(g - c) < 1e-6, name
