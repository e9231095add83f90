"""CPU test of the serving loop's frontier-range allocator (gcsm-bu_b200/csrc/frontier_arena.h),
compiled from its header with a randomised model check."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_frontier_range_allocator(tmp_path):
    exe = str(tmp_path / "arena_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-o", exe, os.path.join(ROOT, "tests", "native", "arena_test.cpp"),
                    "-I", os.path.join(ROOT, "gcsm-bu_b200", "csrc")], check=True)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == "ok", p.stdout + p.stderr
