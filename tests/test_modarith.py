"""Host checks of the device modular arithmetic: modarith.cuh compiled with g++."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "fhe_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_short_montgomery_product_matches_general_form(tmp_path):
    exe = str(tmp_path / "modarith_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, "-o", exe,
                    os.path.join(HERE, "modarith_check.cpp")], check=True)
    for seed in (1, 2):
        out = subprocess.run([exe, "4000000", str(seed)], check=True, capture_output=True, text=True)
        assert out.stdout.strip() == "0"
