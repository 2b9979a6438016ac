"""The reference's own bra executable (oracle/_ref/bra: its main, interpreter,
gate objects and nompi_state, compiled from the reference's sources with
project-written stand-ins for Boost, fmt and cxxopts) on the golden .qcx
programs: its printed output must be what tests/golden/qcx_expected.json
holds, which oracle/bra_ref.py (the Python restatement of bra's interpreter
over the reference's ket calls) produced.  This pins the restatement, and the
rbk-bra interpreter that is tested against the same file, to bra itself.

Two golden programs use instructions the reference's interpreter documents
(docs/bra.md) but rejects: SZn / EXn / CkEXn with a digit count (the digit
check starts one character early, bra/src/interpreter.cpp:2591, :2825, :4252)
and the long forms EXXX... with three or more targets (read_multi_targets_phase
throws when the column count is right, bra/src/interpreter.cpp:1215).  Those
two run with the instructions rewritten to forms bra accepts where one exists;
the failures themselves are checked as bra's behaviour."""
import json
import os
import re
import subprocess

import pytest

from conftest import ROOT
from qcx_compare import same_output, without_timings

BRA = os.path.join(ROOT, "oracle", "_ref", "bra")
GOLDEN = os.path.join(ROOT, "tests", "golden")
needs_bra = pytest.mark.skipif(not os.path.exists(BRA), reason="oracle/_ref/bra is built only where the reference sources are")

# Programs whose every instruction bra accepts as written.
RUNS_AS_WRITTEN = ["fused_brick", "measure_and_events", "events_state_rng", "exit_program", "shor_program",
                   "rotations_adder", "circuits_overlaps", "circuits_tiles", "pauliss_hamiltonian", "pauliss_circuits",
                   "hadamards8"]


def run_bra(exe, text, *args):
    return subprocess.run([exe, *args], input=text, capture_output=True, text=True, timeout=600)


@pytest.fixture(scope="module")
def expected():
    return json.load(open(os.path.join(GOLDEN, "qcx_expected.json")))


@needs_bra
@pytest.mark.parametrize("name", RUNS_AS_WRITTEN)
def test_reference_bra_prints_the_golden_output(expected, name):
    r = run_bra(BRA, open(os.path.join(GOLDEN, "qcx", name + ".qcx")).read())
    assert r.returncode == 0, r.stderr[-2000:]
    same_output(without_timings(r.stdout), without_timings(expected[name]["output"]))


@needs_bra
@pytest.mark.parametrize("instruction,error", [
    ("SZ3 0 1 2", "SZ3 is not supported"),
    ("EX3 0 1 2 0.5", "EX3 is not supported"),
    ("C2EX2 0 1 2 3 0.5", "C2EX2 is not supported"),
    ("EXXX 0 1 2 0.5", "EXXX 0 1 2 0.5"),
    ("EZZZ 0 1 2 0.5", "EZZZ 0 1 2 0.5"),
])
def test_reference_bra_rejects_documented_forms(instruction, error):
    r = run_bra(BRA, f"QUBITS 5\nH 0\n{instruction}\nDO MEASUREMENT\n")
    assert r.returncode != 0
    assert error in r.stderr


@needs_bra
def test_reference_bra_accepts_the_other_long_forms():
    """SZZZ, CCEXX and EXX parse and run (the forms the rewritten programs use)."""
    r = run_bra(BRA, "QUBITS 6\nH 0\nSZZZ 4 5 1\nCCEXX 1 2 4 5 0.3\nEXX 4 5 0.8\nDO MEASUREMENT\n")
    assert r.returncode == 0, r.stderr
    assert "Expectation values of spins:" in r.stdout
