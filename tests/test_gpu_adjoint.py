"""Adjoint gradients (GPU, through the C ABI) against the parameter-shift rule
evaluated with the reference's own ket code (oracle/_ref) where it is built,
else with the C restatement, and against central finite differences.  The
reference has no differentiation support, so these are the checks: energy to
1e-12, parameter-shift gradients to 1e-9, finite differences (h = 1e-6) to 1e-6."""
import math
import os

import numpy as np
import pytest

import oracle
from conftest import ROOT

pytestmark = pytest.mark.gpu

REF_BUILT = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libketref.so"))


def cpu_energy(pkg, n, layers, theta, terms, ref=False):
    ops, _ = pkg.circuits.ansatz(n, layers, thetas=theta)
    o = oracle.KetRef(n) if ref else oracle.COracle(n)
    o.apply(ops)
    return o.expectation(terms).real


@pytest.mark.parametrize("n,layers", [(4, 2), (6, 3), (9, 2)])
def test_adjoint_matches_parameter_shift_and_fd(pkg, n, layers):
    C = pkg.circuits
    terms = C.ansatz_hamiltonian(n)
    _, theta = C.ansatz(n, layers, seed=n)
    spec, nparams = pkg.adjoint.ansatz_spec(n, layers)
    assert nparams == theta.size
    e, g = pkg.adjoint.adjoint_gradient(n, spec, theta, terms)
    assert abs(e - cpu_energy(pkg, n, layers, theta, terms, ref=REF_BUILT)) <= 1e-12
    shift = np.empty_like(theta)
    fd = np.empty_like(theta)
    for k in range(theta.size):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += math.pi / 2
        tm[k] -= math.pi / 2
        shift[k] = 0.5 * (cpu_energy(pkg, n, layers, tp, terms, ref=REF_BUILT) - cpu_energy(pkg, n, layers, tm, terms, ref=REF_BUILT))
        tp, tm = theta.copy(), theta.copy()
        tp[k] += 1e-6
        tm[k] -= 1e-6
        fd[k] = (cpu_energy(pkg, n, layers, tp, terms) - cpu_energy(pkg, n, layers, tm, terms)) / 2e-6
    assert np.abs(g - shift).max() <= 1e-9
    assert np.abs(g - fd).max() <= 1e-6


def test_adjoint_config4_20_qubits(pkg):
    """20-qubit ansatz, 16 layers, 640 parameters: energy against the oracle and
    a sample of gradients against the parameter-shift rule."""
    C = pkg.circuits
    n, layers = 20, 16
    terms = C.ansatz_hamiltonian(n)
    _, theta = C.ansatz(n, layers, seed=1)
    spec, nparams = pkg.adjoint.ansatz_spec(n, layers)
    assert nparams == 640
    e, g = pkg.adjoint.adjoint_gradient(n, spec, theta, terms)
    assert abs(e - cpu_energy(pkg, n, layers, theta, terms)) <= 1e-12
    for k in (0, 19, 20, 333, 620, 639):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += math.pi / 2
        tm[k] -= math.pi / 2
        shift = 0.5 * (cpu_energy(pkg, n, layers, tp, terms) - cpu_energy(pkg, n, layers, tm, terms))
        assert abs(g[k] - shift) <= 1e-9


@pytest.mark.parametrize("n", [7, 13])
def test_adjoint_general_gates_and_c64(pkg, n):
    """Fixed gates of every kind around the rotations (exact inverses in the
    reverse sweep); complex<float> against the FP64 result.  At 13 qubits the
    EX / EY / EZ overlaps come from the two-state Z-sum and pair-sum kernels."""
    C = pkg.circuits
    rng = np.random.default_rng(3)
    spec, k = [], 0
    for _ in range(3):
        for q in range(n):
            spec.append(("U3", (q,), None, 0.0, tuple(rng.uniform(0, 6.28, 3))))
            spec.append((["EX", "EY", "EZ"][q % 3], (q,), k, 0.7, (0.1,)))
            k += 1
        spec += [("CNOT", (0, 3), None, 0.0, ()), ("H", (2,), None, 0.0, ()), ("U", (1, 5), None, 0.0, (3,)),
                 ("SWAP", (4, 6), None, 0.0, ()), ("U1", (6,), None, 0.0, (0.4,)), ("U2", (5,), None, 0.0, (0.3, 1.1)),
                 ("Y", (3,), None, 0.0, ()), ("CZ", (2, 4), None, 0.0, ())]
    theta = rng.uniform(-math.pi, math.pi, k)
    terms = C.ansatz_hamiltonian(n) + [("XYZ" + "I" * (n - 3), 0.3)]
    e, g = pkg.adjoint.adjoint_gradient(n, spec, theta, terms)

    def energy(th):
        ops = []
        for mnem, qubits, param, scale, angles in spec:
            if param is not None:
                ops.append((mnem, qubits, (scale * th[param] + angles[0],)))
            elif mnem == "U":
                ops.append((mnem, qubits, (int(angles[0]),)))
            else:
                ops.append((mnem, qubits, tuple(angles)))
        o = oracle.COracle(n)
        o.apply(ops)
        return o.expectation(terms).real

    assert abs(e - energy(theta)) <= 1e-12
    for j in range(k):
        tp, tm = theta.copy(), theta.copy()
        tp[j] += 1e-6
        tm[j] -= 1e-6
        assert abs(g[j] - (energy(tp) - energy(tm)) / 2e-6) <= 1e-6
    e32, g32 = pkg.adjoint.adjoint_gradient(n, spec, theta, terms, precision=pkg.C64)
    assert abs(e32 - e) <= 1e-5 and np.abs(g32 - g).max() <= 1e-4


def test_autograd_harness_gradcheck(pkg):
    torch = pytest.importorskip("torch")
    n, layers = 4, 2
    terms = pkg.circuits.ansatz_hamiltonian(n)
    spec, nparams = pkg.adjoint.ansatz_spec(n, layers)
    fn = pkg.adjoint.make_autograd_function()
    theta = torch.tensor(np.random.default_rng(0).uniform(-3, 3, nparams), dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda t: fn.apply(t, n, spec, terms), (theta,), eps=1e-6, atol=1e-6)


def test_adjoint_context_reuse_matches_one_shot(pkg):
    """rbk_adjoint_create/run/destroy: repeated gradients on kept state vectors
    equal the one-shot rbk_adjoint_gradient, for several parameter vectors."""
    A, C = pkg.adjoint, pkg.circuits
    n, layers = 12, 3
    spec, k = A.ansatz_spec(n, layers)
    terms = C.ansatz_hamiltonian(n)
    ctx = A.AdjointContext(n)
    try:
        for seed in (1, 2, 3):
            th = np.random.default_rng(seed).uniform(-np.pi, np.pi, size=k)
            e1, g1 = ctx.gradient(spec, th, terms)
            e2, g2 = A.adjoint_gradient(n, spec, th, terms)
            assert e1 == e2 and np.array_equal(g1, g2)
    finally:
        ctx.close()


@pytest.mark.parametrize("precision", ["C128", "C64"])
def test_adjoint_pair_rotate_matches_overlap_path(pkg, monkeypatch, precision):
    """Runs of one-qubit gates in the reverse sweep: the pair-rotate launches
    (overlaps and un-apply in one read and write of both states), with and
    without the owed diagonals and Z-type overlaps folded into their first
    launch, against the path that reads the overlaps first and queues the
    inverses on the engine,
    on the ansatz and on a circuit with fixed gates of every one-qubit kind
    inside the runs (rotations on the low three bits and on high bits, more than
    eleven gates in a run)."""
    A, C = pkg.adjoint, pkg.circuits
    prec = getattr(pkg, precision)
    tol = 1e-12 if precision == "C128" else 2e-5
    rng = np.random.default_rng(11)
    cases = []
    n = 16
    spec, k = A.ansatz_spec(n, 3)
    cases.append((n, spec, rng.uniform(-np.pi, np.pi, k), C.ansatz_hamiltonian(n)))
    n = 14
    spec, k = [], 0
    kinds = ["EX", "EY", "EZ", "H", "U3", "X", "Y", "Z", "U1", "U2"]
    for layer in range(3):
        for q in range(n):
            mnem = kinds[(q + layer) % len(kinds)]
            if mnem in ("EX", "EY", "EZ"):
                spec.append((mnem, (q,), k, 0.5 + 0.1 * layer, (0.2,)))
                k += 1
            elif mnem == "U3":
                spec.append((mnem, (q,), None, 0.0, tuple(rng.uniform(0, 6.28, 3))))
            elif mnem == "U1":
                spec.append((mnem, (q,), None, 0.0, (0.7,)))
            elif mnem == "U2":
                spec.append((mnem, (q,), None, 0.0, (0.3, 1.9)))
            else:
                spec.append((mnem, (q,), None, 0.0, ()))
        spec += [("CNOT", (q, (q + 5) % n), None, 0.0, ()) for q in range(0, n, 3)]
        spec += [("CZ", (q, (q + 1) % n), None, 0.0, ()) for q in range(n)]
    terms = C.ansatz_hamiltonian(n) + [("XYZ" + "I" * (n - 4) + "X", 0.3)]
    cases.append((n, spec, rng.uniform(-np.pi, np.pi, k), terms))
    for n, spec, theta, terms in cases:
        monkeypatch.delenv("RBK_ADJOINT_PAIR_ROTATE", raising=False)
        e2, g2 = A.adjoint_gradient(n, spec, theta, terms, precision=prec)
        monkeypatch.setenv("RBK_ADJOINT_PAIR_ROTATE", "1")
        e1, g1 = A.adjoint_gradient(n, spec, theta, terms, precision=prec)
        monkeypatch.setenv("RBK_ADJOINT_PAIR_ROTATE", "0")
        e0, g0 = A.adjoint_gradient(n, spec, theta, terms, precision=prec)
        monkeypatch.delenv("RBK_ADJOINT_PAIR_ROTATE")
        for e, g in ((e1, g1), (e2, g2)):
            assert abs(e - e0) <= tol
            assert np.abs(g - g0).max() <= tol, (n, np.abs(g - g0).max())
