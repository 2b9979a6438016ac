"""The two 30-qubit workloads at full size against the reference's own output.

tests/golden/full30.npz holds what the reference's ket/bra code (oracle/_ref,
compiled unchanged, IEEE build) gives for
* ``brick``: circuits.brick(30, 20, seed=1, fuse_k=5), the benchmark's circuit;
* ``qft``: circuits.qft_brick(30, 5, seed=1, fuse_k=6);
as size-independent summaries of the 16 GiB state: 2^16 amplitudes at seeded
indices, the 1024 block probabilities over blocks of 2^20 amplitudes, all 90
spins, the energy of H = sum_i Z_i Z_{i+1} + 0.5 sum_i X_i (periodic), and the
overlap with a seeded product state (tests/golden/make_golden30.py).

complex<double>: every summary within 1e-12 of the reference's (the
measurement probabilities of the 1024 blocks among them).
complex<float> (fusion mode 0, gate by gate, and mode 1, the 3xTF32
tensor-core blocks), on the QFT workload: the max amplitude error against the
reference within 2e-5 and 1 - F against the complex<double> state on the GPU
at most 1e-6; the observables, which sum 2^30 float amplitudes, within 1e-4
(spins), 1e-3 (the 60-term energy), 1e-6 (block probabilities and the
product-state overlap, absolute).  The test prints every error.
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


@pytest.mark.parametrize("name", ["brick", "qft"])
def test_c128_matches_reference_at_30_qubits(pkg, golden, name):
    with pkg.State(N, pkg.C128) as s:
        s.apply(circuit(pkg, name))
        got = summaries(pkg, s, golden)
    for key, val in got.items():
        err = np.max(np.abs(val - golden[f"{name}_{key}"]))
        print(f"{name} {key}: max |diff| {err:.3e}")
        assert err <= TOL64, (name, key, err)


def fidelity_between(s64, s128):
    ip, n64, n128 = 0j, 0.0, 0.0
    for off in range(0, 1 << N, CHUNK):
        a = s64.amplitudes(off, CHUNK).astype(np.complex128)
        b = s128.amplitudes(off, CHUNK)
        ip += np.vdot(b, a)
        n64 += np.vdot(a, a).real
        n128 += np.vdot(b, b).real
    return abs(ip) ** 2 / (n64 * n128)


@pytest.mark.parametrize("mode", [0, 1])
def test_c64_qft_brick_against_reference_at_30_qubits(pkg, golden, mode):
    ops = circuit(pkg, "qft")
    with pkg.State(N, pkg.C64) as s64:
        s64.set_fusion_mode(mode)
        s64.apply(ops)
        got = summaries(pkg, s64, golden)
        with pkg.State(N, pkg.C128) as s128:
            s128.apply(ops)
            one_minus_f = 1.0 - fidelity_between(s64, s128)
    want = {k: golden[f"qft_{k}"] for k in got}
    errs = {
        "amps": np.max(np.abs(got["amps"] - want["amps"])),
        "spins": np.max(np.abs(got["spins"] - want["spins"])),
        "energy": abs(got["energy"][0] - want["energy"][0]),
        "overlap": abs(got["product_overlap"][0] - want["product_overlap"][0]),
        "block_probs": np.max(np.abs(got["block_probs"] - want["block_probs"])),
    }
    print(f"mode {mode}:", {k: f"{v:.3e}" for k, v in errs.items()}, f"1-F {one_minus_f:.3e}")
    assert errs["amps"] <= 2e-5
    assert one_minus_f <= 1e-6
    assert errs["spins"] <= 1e-4
    assert errs["energy"] <= 1e-3
    assert errs["overlap"] <= 1e-6
    assert errs["block_probs"] <= 1e-6
