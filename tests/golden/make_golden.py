"""Generates tests/golden/golden.npz + cases.json from the reference itself.

Runs the reference's own ket / bra code (oracle/_ref/libketref.so, built by
oracle/Makefile from the reference sources with the project's Boost shim) on
seeded circuits and records its outputs.  Needs the reference tree at build
time only; the fixtures are committed and the GPU tests read them without it.

    make -C oracle _ref/libketref.so && python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

from __graft_entry__ import load_package  # noqa: E402
import oracle  # noqa: E402

C = load_package().circuits


def ket_test_state(n):
    """Initial state of the reference's own tests
    (ket/test/runtime_gate_numerical.cpp:42-50): a_i = (0.125 (i+1), -0.0625 ((3i+1) mod 7))."""
    i = np.arange(1 << n)
    return 0.125 * (i + 1) - 1j * 0.0625 * ((3 * i + 1) % 7)


def single_gate_cases():
    n = 4
    cases = []
    for q in range(n):
        cases += [("H", (q,), ()), ("X", (q,), ()), ("Y", (q,), ()), ("Z", (q,), ()),
                  ("U1", (q,), (0.7 + q,)), ("U2", (q,), (0.3 + q, 1.9 - q)),
                  ("U3", (q,), (0.4 + q, 2.1 - q, 5.0 + 0.5 * q)),
                  ("EY", (q,), (0.9 - 0.3 * q,)), ("EZ", (q,), (-1.2 + 0.4 * q,))]
    for c in range(n):
        for t in range(n):
            if c != t:
                cases += [("CNOT", (c, t), ()), ("CZ", (c, t), ()), ("SWAP", (c, t), ()),
                          ("U", (c, t), (t + 1,)), ("U", (c, t), (-(c + 1),))]
    return n, cases


def main():
    arrays, meta = {}, {}

    # 1. Every hot-path gate alone on the reference tests' 4-qubit state.
    n, gates = single_gate_cases()
    init = ket_test_state(n)
    outs = []
    for g in gates:
        r = oracle.KetRef(n)
        r.set_amplitudes(init)
        r.apply([g])
        outs.append(r.amplitudes())
    arrays["single_init"] = init
    arrays["single_out"] = np.stack(outs)
    meta["single"] = {"n": n, "ops": gates}

    # 2. Circuits with full outputs (amplitudes, spins, expectation values).
    circuits = {
        "random6": (6, C.random_circuit(6, 300, seed=3)),
        "random9": (9, C.random_circuit(9, 400, seed=11)),
        "brick10_fused5": (10, C.brick(10, 4, seed=2, fuse_k=5)),
        "brick12": (12, C.brick(12, 6, seed=7)),
        "qft_brick8": (8, C.qft_brick(8, 2, seed=4)),
        "ansatz8": (8, C.ansatz(8, 3, seed=5)[0]),
        "hadamards08": (8, [("H", (q,), ()) for q in range(8)]),
    }
    extra_terms = lambda n: [("XYZ" + "I" * (n - 3), 0.3 + 0.1j), ("Y" * n, 1.0), ("Z" * n, -0.25),
                             ("I" * (n - 2) + "XX", 0.5j)]
    for name, (nq, ops) in circuits.items():
        r = oracle.KetRef(nq)
        r.apply(ops)
        arrays[f"{name}_amps"] = r.amplitudes()
        arrays[f"{name}_spins"] = r.spins()
        arrays[f"{name}_energy"] = np.array([r.expectation(C.ansatz_hamiltonian(nq))])
        arrays[f"{name}_pauli"] = np.array([r.expectation(extra_terms(nq))])
        meta[name] = {"n": nq, "ops": ops}

    # 3. The 20-qubit CPU-runnable workload: brick, depth 10 (full state is
    #    16 MiB, so record a fixed sample plus whole-state summaries).
    n20 = 20
    ops20 = C.brick(n20, 10, seed=1)
    r = oracle.KetRef(n20, threads=8)
    r.apply(ops20)
    a = r.amplitudes()
    idx = np.arange(0, 1 << n20, 1021, dtype=np.int64)
    arrays["brick20_idx"] = idx
    arrays["brick20_amps_sample"] = a[idx]
    arrays["brick20_block_probs"] = (np.abs(a) ** 2).reshape(1024, -1).sum(axis=1)
    arrays["brick20_spins"] = r.spins()
    meta["brick20"] = {"n": n20, "generator": "brick(20, 10, seed=1)"}

    # 4. Sampling and measurement on random9 (bra's generator starts at seed 1;
    #    ket::generate_events with a seed builds its own generator).
    n9, ops9 = circuits["random9"]
    r = oracle.KetRef(n9)
    r.apply(ops9)
    arrays["random9_events_seeded"] = r.generate_events(2000, 5)
    r = oracle.KetRef(n9)
    r.apply(ops9)
    arrays["random9_events_state_rng"] = r.generate_events(2000)
    r = oracle.KetRef(n9)
    r.apply(ops9)
    r.seed(23)
    arrays["random9_projective_qubits"] = np.array([2, 5, 8, 0], dtype=np.int64)
    arrays["random9_projective_outcomes"] = np.array(
        [r.projective_measurement(int(q)) for q in arrays["random9_projective_qubits"]], dtype=np.int64)
    arrays["random9_projective_amps"] = r.amplitudes()
    arrays["random9_measure"] = np.array([r.measure()], dtype=np.int64)

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(meta, f, indent=0)
    print("wrote", sorted(arrays))


if __name__ == "__main__":
    main()
