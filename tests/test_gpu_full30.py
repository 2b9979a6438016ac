"""The benchmark's 30-qubit workload at full size against the reference's own output.

tests/golden/full30.npz holds what the reference's ket/bra code (oracle/_ref,
compiled unchanged, IEEE build) gives for ``brick``:
circuits.brick(30, 20, seed=1, fuse_k=5), the benchmark's circuit, as
size-independent summaries of the 16 GiB state: 2^16 amplitudes at seeded
indices, the 1024 block probabilities over blocks of 2^20 amplitudes, all 90
spins, the energy of H = sum_i Z_i Z_{i+1} + 0.5 sum_i X_i (periodic), and the
overlap with a seeded product state (tests/golden/make_golden30.py).

complex<double>: every summary within 1e-12 of the reference's.
"""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(ROOT, "tests", "golden", "full30.npz")
N = 30
LOW = 20
CHUNK = 1 << 24
TOL64 = 1e-12


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


def circuit(pkg, name):
    C = pkg.circuits
    return C.brick(N, 20, seed=1, fuse_k=5) if name == "brick" else C.qft_brick(N, 5, seed=1, fuse_k=6)


def hamiltonian():
    terms = []
    for i in range(N):
        s = ["I"] * N
        s[i] = "Z"
        s[(i + 1) % N] = "Z"
        terms.append(("".join(s), 1.0))
    for i in range(N):
        s = ["I"] * N
        s[i] = "X"
        terms.append(("".join(s), 0.5))
    return terms


def product_state(pkg, precision, a, b):
    p = pkg.State(N, precision)
    for q in range(N):
        p.u3(2.0 * a[q], b[q], 0.0, q)
    return p


def summaries(pkg, s, g):
    """amps at g['idx'], block probabilities, spins, energy, overlap with the product state."""
    idx = g["idx"]
    amps = np.empty(idx.size, dtype=np.complex128)
    probs = np.empty(1 << (N - LOW))
    for off in range(0, 1 << N, CHUNK):
        v = s.amplitudes(off, CHUNK).astype(np.complex128)
        lo, hi = np.searchsorted(idx, [off, off + CHUNK])
        amps[lo:hi] = v[idx[lo:hi] - off]
        probs[off >> LOW:(off + CHUNK) >> LOW] = (np.abs(v.reshape(-1, 1 << LOW)) ** 2).sum(axis=1)
    out = {"amps": amps, "block_probs": probs, "spins": s.spins(),
           "energy": np.array([s.expectation(hamiltonian()).real])}
    with product_state(pkg, s.precision, g["product_a"], g["product_b"]) as p:
        out["product_overlap"] = np.array([s.inner_product(p)])
    return out


@pytest.mark.parametrize("name", ["brick"])
def test_c128_matches_reference_at_30_qubits(pkg, golden, name):
    with pkg.State(N, pkg.C128) as s:
        s.apply(circuit(pkg, name))
        got = summaries(pkg, s, golden)
    for key, val in got.items():
        err = np.max(np.abs(val - golden[f"{name}_{key}"]))
        print(f"{name} {key}: max |diff| {err:.3e}")
        assert err <= TOL64, (name, key, err)
