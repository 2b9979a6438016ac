"""Host logic (CPU, no GPU): the fusion planner's pass programs, executed by a
C++ model of the tile-pass kernel (tests/host/plan_check.cpp), equal the
gates applied one by one; the final layout map is restored to the identity.
The model is built with AddressSanitizer."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT


def test_planner_programs_are_exact(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "plan_check"
    csrc = os.path.join(ROOT, "riken-braket_b200", "csrc")
    # AddressSanitizer: the planner writes fixed-size records; any write past them fails the run
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address", "-fno-omit-frame-pointer", "-I", csrc,
                    "-o", str(exe), os.path.join(ROOT, "tests", "host", "plan_check.cpp"),
                    os.path.join(csrc, "rbk_plan.cpp")],
                   check=True, env={**os.environ, "CXX": "g++"})
    r = subprocess.run([str(exe), "6"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr
    assert "ALL OK" in r.stdout
