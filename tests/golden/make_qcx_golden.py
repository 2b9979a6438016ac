"""Writes tests/golden/qcx/*.qcx (seeded programs that use every instruction the
engine's .qcx interpreter accepts) and their expected results from the
reference: tests/golden/qcx_expected.json (bra's printed output, timing lines
left out) and tests/golden/qcx_golden.npz (final amplitudes).

The expected results come from oracle/bra_ref.py, which executes each program
with the reference's own ket code (oracle/_ref/libketref.so).  Needs the
reference tree at generation time only.

    make -C oracle _ref/libketref.so && python tests/golden/make_qcx_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import bra_ref  # noqa: E402

QCX_DIR = os.path.join(HERE, "qcx")


def a(rng):
    return "%.17g" % rng.uniform(-np.pi, np.pi)


def distinct(rng, n, k):
    return [str(q) for q in rng.choice(n, size=k, replace=False)]


def every_gate(n=6, seed=1):
    """Each gate mnemonic (plain, adjoint, multi-qubit and controlled forms) once,
    interleaved with Hadamard layers so that nothing acts on a basis state."""
    rng = np.random.default_rng(seed)
    L = ["! every gate form of the instruction set", "QUBITS %d" % n]
    L += ["H %d" % q for q in range(n)]
    forms = [
        ("H", 0, 1, 0), ("NOT", 0, 1, 0), ("X", 0, 1, 0), ("XX", 0, 2, 0), ("X3", 0, 3, 0), ("XXX", 0, 3, 0),
        ("Y", 0, 1, 0), ("YY", 0, 2, 0), ("Y3", 0, 3, 0), ("Z", 0, 1, 0), ("ZZ", 0, 2, 0), ("Z3", 0, 3, 0),
        ("SWAP", 0, 2, 0), ("S", 0, 1, 0), ("S+", 0, 1, 0), ("SZ", 0, 1, 0), ("SZ+", 0, 1, 0), ("SZZ", 0, 2, 0),
        ("SZZ+", 0, 2, 0), ("SZ3", 0, 3, 0), ("T", 0, 1, 0), ("T+", 0, 1, 0), ("SX", 0, 1, 0), ("SX+", 0, 1, 0),
        ("SY", 0, 1, 0), ("SY+", 0, 1, 0), ("U1", 0, 1, 1), ("U1+", 0, 1, 1), ("U2", 0, 1, 2), ("U2+", 0, 1, 2),
        ("U3", 0, 1, 3), ("U3+", 0, 1, 3), ("R", 0, 1, "k"), ("R+", 0, 1, "k"), ("U", 0, 2, "k"), ("U+", 0, 2, "k"),
        ("+X", 0, 1, 0), ("-X", 0, 1, 0), ("+Y", 0, 1, 0), ("-Y", 0, 1, 0), ("EX", 0, 1, 1), ("EX+", 0, 1, 1),
        ("EXX", 0, 2, 1), ("EXX+", 0, 2, 1), ("EX3", 0, 3, 1), ("EXXX+", 0, 3, 1), ("EY", 0, 1, 1),
        ("EY+", 0, 1, 1), ("EYY", 0, 2, 1), ("EY3+", 0, 3, 1), ("EZ", 0, 1, 1), ("EZ+", 0, 1, 1),
        ("EZZ", 0, 2, 1), ("EZZZ", 0, 3, 1), ("ESWAP", 0, 2, 1), ("ESWAP+", 0, 2, 1), ("TOFFOLI", 0, 3, 0),
        ("I", 0, 1, 0), ("IC", 0, 1, 0), ("II", 0, 2, 0), ("I3", 0, 3, 0),
        ("CH", 1, 1, 0), ("CCH", 2, 1, 0), ("C3H", 3, 1, 0), ("CNOT", 1, 1, 0), ("CCNOT", 2, 1, 0),
        ("CX", 1, 1, 0), ("C2X2", 2, 2, 0), ("CY", 1, 1, 0), ("CCYY", 2, 2, 0), ("CZ", 1, 1, 0), ("CCZ", 2, 1, 0),
        ("C3Z", 3, 1, 0), ("CZZ", 1, 2, 0), ("CSWAP", 1, 2, 0), ("CCSWAP", 2, 2, 0), ("CS", 1, 1, 0),
        ("CS+", 1, 1, 0), ("CSZZ", 1, 2, 0), ("CT", 1, 1, 0), ("CCT+", 2, 1, 0), ("CSX", 1, 1, 0),
        ("CSX+", 1, 1, 0), ("CSY", 1, 1, 0), ("CCSY+", 2, 1, 0), ("CU1", 1, 1, 1), ("CCU1+", 2, 1, 1),
        ("CU2", 1, 1, 2), ("CU3", 1, 1, 3), ("C2U3+", 2, 1, 3), ("CR", 1, 1, "k"), ("CCR+", 2, 1, "k"),
        ("C+X", 1, 1, 0), ("C-X", 1, 1, 0), ("CC+Y", 2, 1, 0), ("C-Y", 1, 1, 0), ("CEX", 1, 1, 1),
        ("CEX+", 1, 1, 1), ("CEXX", 1, 2, 1), ("C2EY2", 2, 2, 1), ("CEY", 1, 1, 1), ("CEZ", 1, 1, 1),
        ("CCEZ+", 2, 1, 1), ("CEZZ", 1, 2, 1), ("CESWAP", 1, 2, 1), ("CCESWAP+", 2, 2, 1), ("CI", 1, 1, 0),
    ]
    for i, (m, nc, nt, npar) in enumerate(forms):
        qs = distinct(rng, n, nc + nt)
        if npar == "k":
            params = [str(int(rng.integers(1, n + 1)) * (1 if rng.random() < 0.7 else -1))]
        else:
            params = [a(rng) for _ in range(npar)]
        L.append(" ".join([m.lower() if i % 7 == 3 else m] + qs + params))
        if i % 9 == 8:
            L += ["H %d" % q for q in range(n)]
    L += ["DO AMPLITUDES", "DO MEASUREMENT", "DO MEASUREMENT 6", "DO MEASUREMENT -9", "DO MEASUREMENT 0"]
    L += ["EXPECTATION :PAULIS:XZY 4 0 2", "PRINTLN :RESULT", "EXPECTATION :PAULIS:ZZ 1 5", "PRINT :RESULT 1.5 :PI",
          "PRINTLN", "DO AMPLITUDES 0 7 63"]
    return "\n".join(L) + "\n"


def fused_brick(n=11, depth=6, seed=2):
    """Brick layers inside BEGIN/END FUSION blocks, plus blocks that mix in gates
    outside bra's fused set."""
    rng = np.random.default_rng(seed)
    L = ["QUBITS %d" % n, "INITIAL STATE 5"]
    L += ["H %d" % q for q in range(n)]
    for layer in range(depth):
        L.append("BEGIN FUSION")
        for q in range(n):
            L.append("U3 %d %s %s %s" % (q, a(rng), a(rng), a(rng)))
        for q in range(layer % 2, n - 1, 2):
            L.append("CNOT %d %d" % (q, q + 1))
        L.append("U %d %d %d" % (layer % n, (layer + 3) % n, 1 + layer % 4))
        if layer % 3 == 2:
            L += ["+X %d" % (layer % n), "CSX %d %d" % ((layer + 1) % n, (layer + 5) % n),
                  "EZZ %d %d %s" % ((layer + 2) % n, (layer + 7) % n, a(rng))]
        L.append("END FUSION")
    L += ["DO MEASUREMENT 8", "DO AMPLITUDES 1 2 3 1000 2047"]
    return "\n".join(L) + "\n"


def measure_and_events(n=8, seed=3):
    rng = np.random.default_rng(seed)
    L = ["QUBITS %d" % n]
    for q in range(n):
        L += ["H %d" % q, "EY %d %s" % (q, a(rng))]
    for q in range(n - 1):
        L.append("CNOT %d %d" % (q, q + 1))
    L += ["M 3", "PRINTLN :OUTCOME :OUTCOMES:3 :OUTCOMES:0", "M 5", "PRINTLN :OUTCOME",
          "CLEAR 1", "SET 2", "DO MEASUREMENT -8", "U3 0 %s %s %s" % (a(rng), a(rng), a(rng)),
          "GENERATE EVENTS 60 7", "H 0"]
    return "\n".join(L) + "\n"


def events_state_rng(n=9, seed=4):
    rng = np.random.default_rng(seed)
    L = ["QUBITS %d" % n]
    for q in range(n):
        L += ["U3 %d %s %s %s" % (q, a(rng), a(rng), a(rng))]
    L += ["GENERATE EVENTS 40 -1"]
    return "\n".join(L) + "\n"


def exit_program(n=7, seed=5):
    rng = np.random.default_rng(seed)
    L = ["QUBITS %d" % n]
    for q in range(n):
        L += ["H %d" % q, "U1 %d %s" % (q, a(rng)), "+Y %d" % q]
    L += ["EXIT", "H 3"]
    return "\n".join(L) + "\n"


def shor_program():
    """SHORBOX on 7 exponent qubits (base 2, modulus 21), then the inverse QFT of
    the exponent register with H and U+ gates, as in a period-finding circuit."""
    n, nx = 12, 7
    L = ["QUBITS %d" % n, "SHORBOX %d 21 2" % nx]
    top = list(range(n - nx, n))
    for i, j in enumerate(reversed(top)):
        L.append("H %d" % j)
        for k, m in enumerate(reversed(top[:len(top) - 1 - i])):
            L.append("U+ %d %d %d" % (m, j, k + 2))
    L += ["DO MEASUREMENT", "DO AMPLITUDES 0 128 256 4095"]
    return "\n".join(L) + "\n"


def rotations_adder(n=10, seed=6):
    """+X/-X/+Y/-Y state preparation and a QFT-style phase adder (U with positive
    and negative exponents), the instruction mix of bra's adder samples."""
    rng = np.random.default_rng(seed)
    L = ["QUBITS %d" % n, "BIT ASSIGNMENT " + " ".join(str(q) for q in range(n))]
    for q in range(n):
        L.append(["+X", "-X", "+Y", "-Y"][int(rng.integers(4))] + " %d" % q)
    half = n // 2
    for j in range(half, n):
        L.append("H %d" % j)
        for m in range(j + 1, n):
            L.append("U %d %d %d" % (m, j, m - j + 1))
    for j in range(half):
        for m in range(half, n):
            L.append("U %d %d %d" % (j, m, 1 + (m - half + j) % 4))
    for j in reversed(range(half, n)):
        for m in reversed(range(j + 1, n)):
            L.append("U %d %d %d" % (m, j, -(m - j + 1)))
        L.append("H %d" % j)
    L += ["DO MEASUREMENT 5"]
    return "\n".join(L) + "\n"


def bigger_mixed(n=15, seed=7):
    """A 15-qubit program past the per-gate size: tile passes with the wider gate set."""
    rng = np.random.default_rng(seed)
    L = ["QUBITS %d" % n]
    L += ["H %d" % q for q in range(n)]
    for layer in range(4):
        for q in range(n):
            L.append("U3 %d %s %s %s" % (q, a(rng), a(rng), a(rng)))
        L += ["C2EX2 %s %s" % (" ".join(distinct(rng, n, 4)), a(rng)),
              "CCSWAP %s" % " ".join(distinct(rng, n, 4)),
              "ESWAP %s %s" % (" ".join(distinct(rng, n, 2)), a(rng)),
              "EYYY %s %s" % (" ".join(distinct(rng, n, 3)), a(rng)),
              "TOFFOLI %s" % " ".join(distinct(rng, n, 3)),
              "SZZ+ %s" % " ".join(distinct(rng, n, 2)),
              "C3Z %s" % " ".join(distinct(rng, n, 4))]
        for q in range(layer % 2, n - 1, 2):
            L.append("CNOT %d %d" % (q, q + 1))
    L += ["DO MEASUREMENT 10", "EXPECTATION :PAULIS:XZYX 0 5 13 14", "PRINTLN :RESULT"]
    return "\n".join(L) + "\n"


def circuits_overlaps(n=9, seed=8):
    """Three circuits (CIRCUITS 3): pairwise and ALL inner products and fidelities,
    with and without a Pauli operator, a measurement with circuit 2's own seed."""
    rng = np.random.default_rng(seed)

    def layer(L, k):
        for q in range(n):
            L.append("U3 %d %s %s %s" % (q, a(rng), a(rng), a(rng)))
        for q in range(k % 2, n - 1, 2):
            L.append("CNOT %d %d" % (q, q + 1))

    L = ["! several circuits and their overlaps", "CIRCUITS 3", "QUBITS %d" % n]
    L += ["H %d" % q for q in range(n)]
    layer(L, 0)
    L += ["INNERPROD 1", "PRINTLN :RESULT", "INNERPROD 0", "FIDELITY ALL", "PRINTLN :RESULT",
          "INNERPROD 2 :PAULIS:XZY 0 4 8", "PRINTLN :RESULT", "FIDELITY ALL :PAULIS:ZZ 1 2", "PRINTLN :RESULT"]
    L += ["BEGIN CIRCUIT 1"] + ["H %d" % q for q in range(n)]
    layer(L, 1)
    L += ["DO MEASUREMENT 4", "INNERPROD 0", "PRINTLN :RESULT", "FIDELITY ALL", "PRINTLN :RESULT",
          "FIDELITY ALL :PAULIS:ZZ 1 2", "PRINTLN :RESULT", "END CIRCUIT"]
    L += ["BEGIN CIRCUIT 2"] + ["H %d" % q for q in range(0, n, 2)]
    layer(L, 0)
    layer(L, 1)
    L += ["M 3", "PRINTLN :OUTCOME", "FIDELITY ALL", "PRINTLN :RESULT", "INNERPROD 0 :PAULIS:XZY 0 4 8",
          "PRINTLN :RESULT", "FIDELITY ALL :PAULIS:ZZ 1 2", "PRINTLN :RESULT", "DO AMPLITUDES 0 5 77", "END CIRCUIT"]
    return "\n".join(L) + "\n"


def circuits_tiles(n=14, seed=9):
    """Two 14-qubit circuits (tile passes, fusion blocks) compared by FIDELITY and INNERPROD."""
    rng = np.random.default_rng(seed)
    L = ["CIRCUITS 2", "QUBITS %d" % n]
    for k in (0, 1):
        if k:
            L.append("BEGIN CIRCUIT 1")
        L += ["H %d" % q for q in range(n)]
        for layer in range(3):
            L.append("BEGIN FUSION")
            for q in range(n):
                L.append("U3 %d %s %s %s" % (q, a(rng), a(rng), a(rng)))
            L.append("END FUSION")
            for q in range(layer % 2, n - 1, 2):
                L.append("CNOT %d %d" % (q, q + 1))
        L += ["FIDELITY %d" % (1 - k), "PRINTLN :RESULT", "INNERPROD ALL :PAULIS:XYZX 0 3 9 13", "PRINTLN :RESULT",
              "INNERPROD %d" % k, "DO MEASUREMENT 6"]
        if k:
            L.append("END CIRCUIT")
    return "\n".join(L) + "\n"


def _ansatz_lines(n, layers, rng):
    """Config-4 style ansatz: EY and EZ on every qubit, then a CZ ring, per layer."""
    L = []
    for _ in range(layers):
        L += ["EY %d %s" % (q, a(rng)) for q in range(n)]
        L += ["EZ %d %s" % (q, a(rng)) for q in range(n)]
        L += ["CZ %d %d" % (q, (q + 1) % n) for q in range(n)]
    return L


def _string(n, letters):
    s = ["I"] * n
    for q, ch in letters:
        s[q] = ch
    return "".join(s)


def pauliss_hamiltonian(n=10, layers=3, seed=10):
    """PAULISS variables: H = sum Z_i Z_i+1 + 0.5 sum X_i (periodic) built with
    VAR / LET (:=, +=, -=, *=, /=, arrays, :RESULT as a scalar) and read by
    EXPECTATION."""
    rng = np.random.default_rng(seed)
    L = ["! Pauli-string-space variables", "QUBITS %d" % n] + _ansatz_lines(n, layers, rng)
    L += ["VAR H PAULISS", "VAR XS PAULISS 2", "LET H := :PAULIS:%s" % _string(n, [(0, "Z"), (1, "Z")])]
    L += ["LET H += :PAULIS:%s" % _string(n, [(i, "Z"), ((i + 1) % n, "Z")]) for i in range(1, n)]
    L += ["LET XS:0 := :PAULIS:%s" % _string(n, [(0, "X")])]
    L += ["LET XS:0 += :PAULIS:%s" % _string(n, [(i, "X")]) for i in range(1, n)]
    L += ["LET XS:0 *= :COMPLEX:0.5", "let h += xs:0", "EXPECTATION H " + " ".join(str(q) for q in range(n)),
          "PRINTLN :RESULT"]
    L += ["LET XS:1 := H", "LET XS:1 -= :PAULIS:%s" % _string(n, [(0, "Z"), (1, "Z")]), "LET XS:1 /= :COMPLEX:4",
          "LET XS:1 *= :I", "LET XS:1 += :PAULIS:%s" % _string(n, [(2, "Y"), (5, "X"), (7, "Z")]),
          "EXPECTATION XS:1 " + " ".join(str(q) for q in range(n)), "PRINTLN :RESULT"]
    L += ["VAR Q PAULISS", "LET Q := :PAULIS:XZY", "LET Q *= :RESULT", "LET Q -= :PAULIS:ZIX", "LET Q *= :MINUS_I",
          "EXPECTATION Q 3 1 7", "PRINTLN :RESULT", "EXPECTATION :PAULIS:YY 4 6", "PRINTLN :RESULT"]
    L += ["DO MEASUREMENT 6"]
    return "\n".join(L) + "\n"


def pauliss_circuits(n=8, seed=11):
    """PAULISS operators of INNERPROD / FIDELITY over two circuits: a pair whose
    circuits each use their own H, and the ALL form with circuit 0's."""
    rng = np.random.default_rng(seed)
    L = ["CIRCUITS 2", "QUBITS %d" % n] + _ansatz_lines(n, 2, rng)
    L += ["VAR H PAULISS", "LET H := :PAULIS:ZZX", "LET H += :PAULIS:XIY", "LET H *= :COMPLEX:0.75",
          "INNERPROD 1 H 0 3 6", "PRINTLN :RESULT", "FIDELITY ALL H 2 5 7", "PRINTLN :RESULT"]
    L += ["BEGIN CIRCUIT 1"] + _ansatz_lines(n, 2, rng)
    L += ["VAR H PAULISS", "LET H := :PAULIS:YYZ", "LET H -= :PAULIS:IZI", "INNERPROD 0 H 1 2 4", "PRINTLN :RESULT",
          "VAR G PAULISS", "LET G := :PAULIS:XXX", "FIDELITY ALL G 2 5 7", "PRINTLN :RESULT", "END CIRCUIT"]
    return "\n".join(L) + "\n"


PROGRAMS = {
    "every_gate": every_gate,
    "fused_brick": fused_brick,
    "measure_and_events": measure_and_events,
    "events_state_rng": events_state_rng,
    "exit_program": exit_program,
    "shor_program": shor_program,
    "rotations_adder": rotations_adder,
    "bigger_mixed": bigger_mixed,
    "circuits_overlaps": circuits_overlaps,
    "circuits_tiles": circuits_tiles,
    "pauliss_hamiltonian": pauliss_hamiltonian,
    "pauliss_circuits": pauliss_circuits,
    "hadamards8": lambda: "QUBITS 8\n" + "".join("H %d\n" % q for q in range(8)) + "DO MEASUREMENT\n",
}


def main():
    os.makedirs(QCX_DIR, exist_ok=True)
    expected, arrays = {}, {}
    for name, make in PROGRAMS.items():
        text = make()
        with open(os.path.join(QCX_DIR, name + ".qcx"), "w") as f:
            f.write(text)
        out, amps, _ = bra_ref.run(text)
        ends_with_events = "Events:" in out
        expected[name] = {"output": out, "amplitudes": not ends_with_events}
        if not ends_with_events:  # the reference overwrites the state with prefix sums for events
            arrays[name] = amps
    with open(os.path.join(HERE, "qcx_expected.json"), "w") as f:
        json.dump(expected, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "qcx_golden.npz"), **arrays)
    print("wrote", sorted(expected))


if __name__ == "__main__":
    main()
