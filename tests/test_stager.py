"""The serving loop's threaded host copies (evora_b200/csrc/stager.h),
compiled on its own with the host compiler: it holds no CUDA code."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_stager_copies(tmp_path):
    exe = tmp_path / "stager_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", os.path.join(HERE, "native", "stager_check.cpp"),
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
