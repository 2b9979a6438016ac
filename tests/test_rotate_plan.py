"""Host logic (CPU, no GPU): the adjoint sweep's pair-rotate launches planned by
rbk::plan_rotations, executed by a C++ model of pair_rotate_kernel
(tests/host/rotate_check.cpp) -- owed diagonal, Z sums, register phases through
the swizzled shared-memory slots, overlaps and gates -- equal the gates applied
one by one, with the overlaps and Z sums taken directly; phase exchanges behind
a warp barrier read back only slots the same warp wrote.  The model is built
with AddressSanitizer."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT


def test_pair_rotate_plans_are_exact(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "rotate_check"
    csrc = os.path.join(ROOT, "riken-braket_b200", "csrc")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address", "-fno-omit-frame-pointer", "-I", csrc,
                    "-I", cuda_inc, "-o", str(exe), os.path.join(ROOT, "tests", "host", "rotate_check.cpp"),
                    os.path.join(csrc, "rbk_rotate_plan.cpp")], check=True)
    r = subprocess.run([str(exe), "80"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr
    assert "ALL OK" in r.stdout
