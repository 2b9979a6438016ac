"""Generates tests/golden/full30.npz: the reference's own outputs for the two
30-qubit complex<double> workloads at full size.

* ``brick``: ``circuits.brick(30, 20, seed=1, fuse_k=5)``, the circuit the
  benchmark times (H layer, 20 layers of seeded U3 and CNOT pairs, BEGIN/END
  FUSION blocks of <= 5 qubits).
* ``qft``: ``circuits.qft_brick(30, 5, seed=1, fuse_k=6)`` (H j then U m j (m-j+1)
  for every m > j, then 5 seeded brick layers, fusion blocks of 6).

Both run through oracle/_ref/libketref.so, the reference's ket headers and
bra fused-gate sources compiled unchanged (IEEE -O2 build, OpenMP threads).
A 2^30-amplitude state is 16 GiB, so the script records size-independent
summaries instead of the vector:

* 2^16 amplitudes at seeded distinct indices (``idx``, shared by both circuits);
* the 1024 block probabilities sum_{i in block b} |a_i|^2 (blocks of 2^20);
* all 90 spins (ket::ranges::all_spin_expectation_values);
* the energy of H = sum_i Z_i Z_{i+1} + 0.5 sum_i X_i (periodic), term by term
  with bra's EXPECTATION :PAULIS: on the operated qubits;
* the overlap <P|psi> with the seeded product state
  P = (x)_q (cos a_q |0> + e^{i b_q} sin a_q |1>), which a GPU test builds
  with U3(2 a_q, b_q, 0) on every qubit and reads with one inner product.

Needs about 40 GiB of host memory and roughly an hour on 8 cores.  Run from the
repository root after ``make -C oracle _ref/libketref.so``:

    python tests/golden/make_golden30.py [brick|qft ...]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

from __graft_entry__ import load_package  # noqa: E402
import oracle  # noqa: E402

C = load_package().circuits

N = 30
SAMPLE_SEED = 30
PRODUCT_SEED = 31
NUM_SAMPLES = 1 << 16
LOW = 20  # block probabilities over blocks of 2^LOW amplitudes


def workloads():
    return {
        "brick": C.brick(N, 20, seed=1, fuse_k=5),
        "qft": C.qft_brick(N, 5, seed=1, fuse_k=6),
    }


def sample_indices():
    rng = np.random.Generator(np.random.PCG64(SAMPLE_SEED))
    return np.sort(rng.choice(1 << N, size=NUM_SAMPLES, replace=False)).astype(np.int64)


def product_angles():
    """(a_q, b_q) for q = 0..N-1: a uniform [0, pi/2), b uniform [0, 2 pi)."""
    rng = np.random.Generator(np.random.PCG64(PRODUCT_SEED))
    a = rng.uniform(0.0, 0.5 * np.pi, size=N)
    b = rng.uniform(0.0, 2.0 * np.pi, size=N)
    return a, b


def product_vector(a, b, qubits):
    """Amplitudes of (x)_{q in qubits} (cos a_q|0> + e^{i b_q} sin a_q|1>),
    index bit j <-> qubits[j]."""
    v = np.ones(1, dtype=np.complex128)
    for q in qubits:
        f = np.array([np.cos(a[q]), np.exp(1j * b[q]) * np.sin(a[q])])
        v = np.concatenate([v * f[0], v * f[1]])  # new bit is the highest so far
    return v


def summaries(name, ops, idx, a_prod, b_prod, threads):
    out = {}
    t0 = time.time()
    r = oracle.KetRef(N, threads=threads)
    r.apply(ops)
    t1 = time.time()
    print(f"{name}: circuit {t1 - t0:.0f} s", flush=True)
    out["spins"] = r.spins()
    energy = 0.0
    for i in range(N):
        energy += r.expectation_on("ZZ", [i, (i + 1) % N]).real
    for i in range(N):
        energy += 0.5 * r.expectation_on("X", [i]).real
    out["energy"] = np.array([energy])
    t2 = time.time()
    print(f"{name}: spins + energy {t2 - t1:.0f} s", flush=True)
    amps = r.amplitudes()
    del r
    out["amps"] = amps[idx]
    A = amps.reshape(1 << (N - LOW), 1 << LOW)
    probs = np.empty(A.shape[0])
    for r0 in range(0, A.shape[0], 16):
        blk = A[r0:r0 + 16]
        probs[r0:r0 + 16] = (blk.real ** 2 + blk.imag ** 2).sum(axis=1)
    out["block_probs"] = probs
    p_lo = product_vector(a_prod, b_prod, range(LOW))
    p_hi = product_vector(a_prod, b_prod, range(LOW, N))
    out["product_overlap"] = np.array([np.conj(p_hi) @ (A @ np.conj(p_lo))])
    print(f"{name}: summaries {time.time() - t2:.0f} s; norm {probs.sum():.15f} energy {energy:.15f}", flush=True)
    return out


def main():
    names = sys.argv[1:] or ["brick", "qft"]
    threads = os.cpu_count() or 1
    path = os.path.join(HERE, "full30.npz")
    arrays = dict(np.load(path)) if os.path.exists(path) else {}
    idx = sample_indices()
    a_prod, b_prod = product_angles()
    arrays["idx"] = idx
    arrays["product_a"], arrays["product_b"] = a_prod, b_prod
    wl = workloads()
    for name in names:
        for key, val in summaries(name, wl[name], idx, a_prod, b_prod, threads).items():
            arrays[f"{name}_{key}"] = val
        np.savez_compressed(path, **arrays)
        print("wrote", path, sorted(arrays), flush=True)


if __name__ == "__main__":
    main()
