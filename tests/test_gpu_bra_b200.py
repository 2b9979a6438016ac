"""bra itself on the B200: riken-braket_b200/bin/bra-b200 is the reference's
bra (its main, interpreter and gate objects, compiled from the reference's
sources) with this project's bra::nompi_state, whose amplitudes live in HBM
and whose do_* backend calls the engine's C ABI.  It must print what the
reference's own bra prints for the same .qcx text: the golden programs
against tests/golden/qcx_expected.json and, where the reference's CPU build
(oracle/_ref/bra) is at hand, against its output run for run; a 20-qubit
fused brick, a program of bra's classical layer (VAR/LET/@label/JUMPIF with
variables as gate operands) and a depolarizing-channel run, each against the
reference's CPU run; the instructions the reference rejects, rejected with
the same message."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from qcx_compare import same_output, without_timings
from test_bra_reference import RUNS_AS_WRITTEN

pytestmark = pytest.mark.gpu

B200 = os.path.join(ROOT, "riken-braket_b200", "bin", "bra-b200")
REF = os.path.join(ROOT, "oracle", "_ref", "bra")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def run(exe, text, *args):
    return subprocess.run([exe, *args], input=text, capture_output=True, text=True, timeout=900)


@pytest.fixture(scope="module")
def expected():
    if not os.path.exists(B200):
        pytest.fail("riken-braket_b200/bin/bra-b200 is not built (make -C riken-braket_b200/bra)")
    return json.load(open(os.path.join(GOLDEN, "qcx_expected.json")))


@pytest.mark.parametrize("name", RUNS_AS_WRITTEN)
def test_bra_b200_prints_the_reference_output(expected, name):
    text = open(os.path.join(GOLDEN, "qcx", name + ".qcx")).read()
    r = run(B200, text)
    assert r.returncode == 0, r.stderr[-2000:]
    got = without_timings(r.stdout)
    same_output(got, without_timings(expected[name]["output"]))
    if os.path.exists(REF):
        ref = run(REF, text)
        assert ref.returncode == 0
        same_output(got, without_timings(ref.stdout))


def brick_program(n, depth, seed):
    """A U3 on every qubit, then CNOTs on alternating neighbour pairs, each
    pair of CNOTs and the four qubits' U3s as one fusion block.  Blocks stay
    small: the reference's cache-aware build (16 on-cache qubits) assumes a
    block operates on fewer qubits than that."""
    rng = np.random.default_rng(seed)
    lines = [f"QUBITS {n}"] + [f"H {q}" for q in range(n)]

    def u3(q):
        t, p, l = rng.uniform(0.0, 6.283185307179586, 3)
        return f"U3 {q} {float(t)!r} {float(p)!r} {float(l)!r}"

    for layer in range(depth):
        pairs = [(q, q + 1) for q in range(layer % 2, n - 1, 2)]
        covered = {q for pr in pairs for q in pr}
        lines += [u3(q) for q in range(n) if q not in covered]
        for i in range(0, len(pairs), 2):
            group = pairs[i:i + 2]
            lines.append("BEGIN FUSION")
            lines += [u3(q) for pr in group for q in pr]
            lines += [f"CNOT {a} {b}" for a, b in group]
            lines.append("END FUSION")
    lines += ["DO MEASUREMENT", "EXPECTATION :PAULIS:ZXZ 0 5 9", "PRINT :RESULT", "DO AMPLITUDES 0 1 77 1023"]
    return "\n".join(lines) + "\n"


def test_bra_b200_20_qubit_fused_brick_matches_reference_bra(expected):
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/bra was not built")
    text = brick_program(20, 10, 7)
    got, ref = run(B200, text), run(REF, text, "--threads", str(os.cpu_count() or 1))
    assert got.returncode == 0 and ref.returncode == 0, got.stderr[-2000:] + ref.stderr[-2000:]
    same_output(without_timings(got.stdout), without_timings(ref.stdout))


CLASSICAL = """QUBITS 6
VAR K INT
VAR TH REAL
VAR ACC COMPLEX
LET K := 0
LET TH := 0.3
H 0
H 1
@LOOP
U3 0 TH 0.2 0.1
CNOT 0 1
EZ 2 TH
CNOT 1 2
LET TH *= 1.5
LET K += 1
JUMPIF LOOP K < 4
M 1
PRINTLN K TH :OUTCOME
VAR OP PAULISS
LET OP := :PAULIS:ZZX
EXPECTATION OP 0 1 2
LET ACC := :RESULT
PRINTLN ACC
DO MEASUREMENT
"""

DEPOLARIZING = """QUBITS 8
DEPOLARIZING CHANNEL P_X=0.05,P_Y=0.04,P_Z=0.03,SEED=17
H 0
CNOT 0 1
U3 2 0.7 0.1 0.2
BEGIN FUSION
U3 3 0.4 0.5 0.6
CNOT 3 4
CZ 4 5
END FUSION
T 6
CNOT 6 7
DO MEASUREMENT 6
DO AMPLITUDES 0 3 17 255
"""


@pytest.mark.parametrize("name,text,args", [
    ("classical", CLASSICAL, ()), ("classical_seed5", CLASSICAL, ("--seed", "5")),
    ("depolarizing", DEPOLARIZING, ()), ("depolarizing_own_seed", DEPOLARIZING.replace("SEED=17", "SEED=-1"), ("--seed", "3")),
])
def test_bra_b200_classical_layer_and_noise_match_reference_bra(expected, name, text, args):
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/bra was not built")
    got, ref = run(B200, text, *args), run(REF, text, *args)
    assert got.returncode == 0 and ref.returncode == 0, got.stderr[-2000:] + ref.stderr[-2000:]
    same_output(without_timings(got.stdout), without_timings(ref.stdout))


@pytest.mark.parametrize("instruction", ["SZ3 0 1 2", "EX3 0 1 2 0.5", "C2EX2 0 1 2 3 0.5", "EXXX 0 1 2 0.5"])
def test_bra_b200_rejects_what_bra_rejects(expected, instruction):
    text = f"QUBITS 5\nH 0\n{instruction}\nDO MEASUREMENT\n"
    got = run(B200, text)
    assert got.returncode != 0
    if os.path.exists(REF):
        ref = run(REF, text)
        assert ref.returncode != 0
        assert got.stderr.strip().splitlines()[-1] == ref.stderr.strip().splitlines()[-1]
