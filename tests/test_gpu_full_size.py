"""The configurations at their full sizes, where no CPU oracle finishes in
seconds, through size-independent properties: a circuit followed by its exact
inverse returns |0...0> (every amplitude, through the fused passes and the
layout map), and the norm is preserved after the forward circuit.  Errors:
c128 <= 1e-10 on the |0> amplitude and 1e-12 on the norm (depth ~40 of FP64
rounding), c64 <= 2e-4 and 2e-5."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def free_gib():
    free, _ = torch.cuda.mem_get_info()
    return free / 2**30


def round_trip(pkg, n, precision, ops, tol_amp, tol_norm):
    with pkg.State(n, precision) as s:
        s.apply(ops)
        norm = s.norm2()
        s.apply(pkg.circuits.inverse(ops))
        a0 = s.amplitudes(0, 1)[0]
        tail = s.probabilities(1, 4095).sum()
    assert abs(norm - 1.0) <= tol_norm
    assert abs(complex(a0) - 1.0) <= tol_amp
    assert tail <= tol_amp


def test_brick30_c128_round_trip(pkg):
    ops = pkg.circuits.brick(30, 20, seed=1, fuse_k=5)
    round_trip(pkg, 30, pkg.C128, ops, 1e-10, 1e-12)


def test_qft_brick32_c64_round_trip(pkg):
    ops = pkg.circuits.qft_brick(32, 5, seed=1, fuse_k=6)
    round_trip(pkg, 32, pkg.C64, ops, 2e-4, 2e-5)


def test_qft_brick32_c64_tensor_core_round_trip(pkg):
    ops = pkg.circuits.qft_brick(32, 5, seed=1, fuse_k=6)
    with pkg.State(32, pkg.C64) as s:
        s.set_fusion_mode(1)
        s.apply(ops)
        norm = s.norm2()
        s.apply(pkg.circuits.inverse(ops))
        a0 = s.amplitudes(0, 1)[0]
    assert abs(norm - 1.0) <= 2e-4
    assert abs(complex(a0) - 1.0) <= 5e-4


def test_qft_brick33_c128_round_trip(pkg):
    if free_gib() < 140:
        pytest.skip("needs 128 GiB of free device memory")
    ops = pkg.circuits.qft_brick(33, 5, seed=1, fuse_k=6)
    round_trip(pkg, 33, pkg.C128, ops, 1e-10, 1e-12)
