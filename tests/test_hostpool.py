"""The host copy pool of pageable queries (csrc/hostpool.h), built with g++
and run on the CPU: parts of a job run once each, jobs follow one another on
one pool, and pool_copy moves every byte of its segments."""
import pathlib
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_hostpool(tmp_path):
    exe = tmp_path / "hostpool_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-I", str(ROOT / "illuminaprt_b200" / "csrc"),
                    str(ROOT / "tests" / "hostpool_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "hostpool ok" in r.stdout
