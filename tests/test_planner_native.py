"""CPU test of the planner (gcsm-bu_b200/csrc/plan.cpp), compiled from its sources with a
harness that checks order invariants and the Cartesian-tail polynomial against brute force."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gcsm-bu_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_plans_and_tail_polynomial(tmp_path):
    exe = str(tmp_path / "plan_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-o", exe, os.path.join(ROOT, "tests", "native", "plan_test.cpp"),
                    os.path.join(CSRC, "plan.cpp"), os.path.join(CSRC, "query.cpp"), "-I", CSRC], check=True)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0 and p.stdout.startswith("ok"), p.stdout + p.stderr
