"""The C-ABI library (CPU, no GPU): it loads, exports every function that
include/rbk.h declares, and fails loudly -- with a status, not a crash -- when
no GPU is present."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "rbk.h")
LIB = os.path.join(ROOT, "riken-braket_b200", "librbk.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(rbk_[a-z_0-9]+)\s*\(", text, flags=re.M)))


def test_header_declares_the_api():
    names = declared_functions()
    for required in ("rbk_state_create", "rbk_phase_shift3", "rbk_pauli_x", "rbk_spin_expectation_values",
                     "rbk_expectation_pauli", "rbk_inner_product", "rbk_begin_fusion", "rbk_end_fusion"):
        assert required in names
    assert len(names) >= 40


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "librbk.so is not built"
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_pass_descriptor_bytes(pkg):
    """The fused pass's by-value parameter block fits CUDA's 32 KB kernel
    parameter limit (bench.py counts it as the host->device bytes of a pass)."""
    b = pkg.rbk.pass_descriptor_bytes()
    assert 16384 <= b <= 32764


def test_no_gpu_is_a_clean_error(pkg):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(pkg.RbkError) as e:
        pkg.State(4)
    assert e.value.code == 2  # RBK_ERR_CUDA
