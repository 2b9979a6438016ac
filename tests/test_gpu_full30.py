"""The 30-qubit workloads at full size against the reference's own outputs.

tests/golden/full30.npz holds what the reference (ket + bra's fused gates,
oracle/_ref) computed for

* the benchmark's brick circuit, brick(30, 20, seed=1, fuse_k=5), and
* the QFT + brick circuit, qft_brick(30, 5, seed=1, fuse_k=6),

in complex<double> (tests/golden/make_golden30.py): 2^16 amplitudes at seeded
indices, the 1024 block probabilities (blocks of 2^20 amplitudes), all 90
spins, the energy of H = sum Z_i Z_i+1 + 0.5 sum X_i, and the overlap with a
seeded product state.  The complex<double> engine must match every field to
1e-12 (absolute).  complex<float>, gate by gate and with 5-6 qubit fusion
blocks as 3xTF32 tensor-core GEMMs, is compared with the same fixture
(max amplitude error <= 2e-5, overlap error <= 1e-6 relative) and with the
complex<double> engine state on the full vector (1 - fidelity <= 1e-6).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "full30.npz")
N = 30
TOL64 = 1e-12
CHUNK = 1 << 24


@pytest.fixture(scope="module")
def full30():
    if not os.path.exists(FIXTURE):
        pytest.fail("tests/golden/full30.npz is missing (tests/golden/make_golden30.py writes it)")
    return dict(np.load(FIXTURE))


def workload(pkg, name):
    C = pkg.circuits
    return C.brick(N, 20, seed=1, fuse_k=5) if name == "brick" else C.qft_brick(N, 5, seed=1, fuse_k=6)


def summaries(pkg, s, fix):
    """The fixture's fields, read from an engine state."""
    idx = fix["idx"]
    amps = np.empty(idx.size, dtype=np.complex128)
    probs = np.zeros(1 << (N - 20))
    for off in range(0, 1 << N, CHUNK):
        chunk = s.amplitudes(off, CHUNK).astype(np.complex128)
        sel = (idx >= off) & (idx < off + CHUNK)
        amps[sel] = chunk[idx[sel] - off]
        probs[off >> 20:(off + CHUNK) >> 20] = (chunk.real ** 2 + chunk.imag ** 2).reshape(-1, 1 << 20).sum(axis=1)
    out = {"amps": amps, "block_probs": probs, "spins": s.spins(),
           "energy": np.array([s.expectation(pkg.circuits.ansatz_hamiltonian(N)).real])}
    prod = pkg.State(N, s.precision)
    prod.apply([("U3", (q,), (2.0 * float(fix["product_a"][q]), float(fix["product_b"][q]), 0.0)) for q in range(N)])
    out["product_overlap"] = np.array([s.inner_product(prod)])  # <P|psi>
    prod.close()
    return out


def errors(got, fix, name):
    return {k: float(np.abs(got[k] - fix[f"{name}_{k}"]).max()) for k in got}


@pytest.mark.parametrize("name", ["brick", "qft"])
def test_c128_matches_reference_at_30_qubits(pkg, full30, name):
    s = pkg.State(N, pkg.C128)
    s.apply(workload(pkg, name))
    err = errors(summaries(pkg, s, full30), full30, name)
    s.close()
    print(name, "complex<double> errors against the reference:", err)
    for k, e in err.items():
        assert e <= TOL64, (name, k, e)


def _fidelity(a, b):
    """|<a|b>|^2 / (<a|a><b|b>) over the full vectors, read in chunks."""
    ab, aa, bb = 0j, 0.0, 0.0
    for off in range(0, 1 << N, CHUNK):
        x = a.amplitudes(off, CHUNK).astype(np.complex128)
        y = b.amplitudes(off, CHUNK).astype(np.complex128)
        ab += np.vdot(x, y)
        aa += np.vdot(x, x).real
        bb += np.vdot(y, y).real
    return abs(ab) ** 2 / (aa * bb)


@pytest.mark.parametrize("mode", [0, 1], ids=["gate-by-gate", "tensor-core-blocks"])
def test_c64_qft_brick_against_reference_at_30_qubits(pkg, full30, mode):
    ops = workload(pkg, "qft")
    s = pkg.State(N, pkg.C64)
    s.set_fusion_mode(mode)
    s.apply(ops)
    got = summaries(pkg, s, full30)
    err = errors(got, full30, "qft")
    rel_overlap = err["product_overlap"] / abs(full30["qft_product_overlap"][0])
    ref = pkg.State(N, pkg.C128)
    ref.apply(ops)
    infidelity = 1.0 - _fidelity(ref, s)
    ref.close()
    s.close()
    print(f"complex<float> mode {mode} against the reference: max |da| {err['amps']:.3e}, "
          f"overlap error {err['product_overlap']:.3e} ({rel_overlap:.3e} relative), spins {err['spins']:.3e}, "
          f"energy {err['energy']:.3e}; 1 - F against complex<double> {infidelity:.3e}")
    assert err["amps"] <= 2e-5
    assert rel_overlap <= 1e-6
    assert err["spins"] <= 1e-5 and err["energy"] <= 1e-4
    assert infidelity <= 1e-6
