"""Batched energies and adjoint gradients (rbk_batch_*): every instance of a
mixed-size batch against the engine's single-instance adjoint sweep, the
parameter-shift rule on the reference ket code for a few instances, and
complex<float> against FP64."""
import math
import os

import numpy as np
import pytest

import oracle
from conftest import ROOT

pytestmark = pytest.mark.gpu
REF_BUILT = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libketref.so"))


def mixed_batch(pkg, sizes, seed=5):
    A, C = pkg.adjoint, pkg.circuits
    rng = np.random.default_rng(seed)
    inst, thetas = [], []
    for i, n in enumerate(sizes):
        layers = 2 + i % 3
        spec, k = A.ansatz_spec(n, layers)
        if i % 4 == 1:  # a few fixed gates of other kinds in the mix
            spec = [("H", (0,), None, 0.0, ()), ("U3", (1 % n,), None, 0.0, (0.3, 1.1, -0.7)),
                    ("CNOT", (0, n - 1), None, 0.0, ()), ("U", (1 % n, 0), None, 0.0, (3,))] + spec + [
                    ("EX", (n - 1,), k - 1, 0.5, (0.2,)), ("SWAP", (0, n - 1), None, 0.0, ())]
        inst.append((n, spec, k, C.ansatz_hamiltonian(n)))
        thetas.append(rng.uniform(-math.pi, math.pi, size=k))
    return inst, thetas


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_single_instance_adjoint(pkg, precision):
    A = pkg.adjoint
    sizes = [3, 12, 5, 13, 8, 10, 4, 11, 7, 9, 6, 14, 12, 2 + 1]
    inst, thetas = mixed_batch(pkg, sizes)
    b = A.Batch(inst, precision=precision)
    try:
        energies, grads = b.run(thetas)
        st = b.stats()
        assert st["num_small"] + st["num_large"] == len(sizes)
        assert st["num_large"] == (1 if precision == 1 else 2)  # 14 (and 13 for c128) exceed shared memory
        assert st["threads"] in (128, 256, 512, 1024)
        tol = 1e-10 if precision == 0 else 2e-4
        for (n, spec, k, terms), th, e, g in zip(inst, thetas, energies, grads):
            e_ref, g_ref = A.adjoint_gradient(n, spec, th, terms)
            assert abs(e - e_ref) <= tol * max(1.0, abs(e_ref)), n
            assert np.abs(g - g_ref).max() <= tol * max(1.0, np.abs(g_ref).max()), n
        # replayed graph: same numbers, new parameters change them
        e2, g2 = b.run(thetas)
        assert np.array_equal(e2, energies) and all(np.array_equal(x, y) for x, y in zip(g2, grads))
        e3, _ = b.run([t + 0.1 for t in thetas])
        assert not np.allclose(e3, energies)
    finally:
        b.close()


@pytest.mark.skipif(not REF_BUILT, reason="oracle/_ref not built (needs the reference sources)")
def test_batch_gradients_vs_parameter_shift_on_reference(pkg):
    """dE/dtheta_k = [E(theta_k + pi/2) - E(theta_k - pi/2)] / 2 for RY/RZ (= EY/EZ with
    scale -1/2), each E evaluated with the reference ket code."""
    A, C = pkg.adjoint, pkg.circuits
    sizes = [6, 9, 11]
    inst, thetas = [], []
    for i, n in enumerate(sizes):
        spec, k = A.ansatz_spec(n, 2)
        inst.append((n, spec, k, C.ansatz_hamiltonian(n)))
        thetas.append(np.random.default_rng(10 + i).uniform(-math.pi, math.pi, size=k))
    b = A.Batch(inst)
    energies, grads = b.run(thetas)
    b.close()
    for (n, spec, k, terms), th, e, g in zip(inst, thetas, energies, grads):
        def energy(t):
            r = oracle.KetRef(n)
            r.apply(C.ansatz(n, 2, thetas=t)[0])
            return r.expectation(terms).real
        assert abs(e - energy(th)) <= 1e-10
        for j in range(0, k, 3):
            tp, tm = th.copy(), th.copy()
            tp[j] += math.pi / 2
            tm[j] -= math.pi / 2
            assert abs(g[j] - 0.5 * (energy(tp) - energy(tm))) <= 1e-9


def test_config5_sample(pkg):
    """A 64-instance sample of the config-5 draw (n log-uniform in [10, 24],
    depth U{4..16}, per-instance seeds), restricted to n <= 16 so that the
    single-instance reference sweep stays quick."""
    A, C = pkg.adjoint, pkg.circuits
    draws = [d for d in C.batch_instances(400) if d[0] <= 16][:64]
    inst, thetas = [], []
    for n, layers, th in draws:
        spec, k = A.ansatz_spec(n, layers)
        inst.append((n, spec, k, C.ansatz_hamiltonian(n)))
        thetas.append(th)
    b = A.Batch(inst)
    energies, grads = b.run(thetas)
    b.close()
    for i in range(0, len(inst), 7):
        n, spec, k, terms = inst[i]
        e_ref, g_ref = A.adjoint_gradient(n, spec, thetas[i], terms)
        assert abs(energies[i] - e_ref) <= 1e-10
        assert np.abs(grads[i] - g_ref).max() <= 1e-10
