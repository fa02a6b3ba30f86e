"""The host thread pool that walks the framing of a batch of compressed
chunks in parallel (dials_metal_spotfinder_b200/csrc/sf_pool.hh), built
from tests/cpp/pool_check.cc with the host compiler and run on the CPU."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_pool_runs_every_item_once_and_passes_exceptions_on(tmp_path):
    exe = tmp_path / "pool_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-o", str(exe),
                    os.path.join(ROOT, "tests", "cpp", "pool_check.cc")], check=True)
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == "ok"
