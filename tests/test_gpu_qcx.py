"""bra's .qcx programs end to end on the GPU (rbk_qcx_run and bin/rbk-bra)
against the reference's results for the same text (tests/golden/qcx_*,
produced by running the reference ket code through oracle/bra_ref.py).

Printed numbers are compared to within one unit of the last printed digit
(bra prints 3 to 9 digits; a value at a rounding boundary or a signed zero may
print differently), event indices and measurement results exactly, and the
final state to 1e-12 (c128) max amplitude error."""
import glob
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from qcx_compare import same_output

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(ROOT, "tests", "golden")
PROGRAMS = sorted(glob.glob(os.path.join(GOLDEN, "qcx", "*.qcx")))
TOL64 = 1e-12


@pytest.fixture(scope="module")
def expected():
    return json.load(open(os.path.join(GOLDEN, "qcx_expected.json"))), dict(np.load(os.path.join(GOLDEN, "qcx_golden.npz")))


@pytest.mark.parametrize("path", PROGRAMS, ids=os.path.basename)
def test_program_vs_reference(pkg, expected, path):
    exp, arrays = expected
    name = os.path.basename(path)[:-4]
    out, state = pkg.qcx.run(open(path).read(), keep_state=True)
    with state:
        same_output(out, exp[name]["output"])
        if exp[name]["amplitudes"]:
            assert np.abs(state.amplitudes() - arrays[name]).max() <= TOL64


@pytest.mark.parametrize("name", ["fused_brick", "bigger_mixed", "every_gate"])
def test_unfused_execution_agrees(pkg, expected, name):
    exp, arrays = expected
    out, state = pkg.qcx.run(open(os.path.join(GOLDEN, "qcx", name + ".qcx")).read(), deferred=False, keep_state=True)
    with state:
        same_output(out, exp[name]["output"])
        assert np.abs(state.amplitudes() - arrays[name]).max() <= TOL64


def test_timing_lines_follow_bra(pkg, expected):
    exp, _ = expected
    text = open(os.path.join(GOLDEN, "qcx", "measure_and_events.qcx")).read()
    out, _ = pkg.qcx.run(text, timing=True)
    timing = re.compile(r"^(Operations|Expectation values|Events|Amplitudes|Measurement) finished: \S+ \(\S+\)$")
    lines = out.splitlines()
    assert sum(bool(timing.match(line)) for line in lines) == 4
    same_output("\n".join(line for line in lines if not timing.match(line)) + "\n", exp["measure_and_events"]["output"])


def test_c64_program_within_float_tolerance(pkg, expected):
    exp, arrays = expected
    out, state = pkg.qcx.run(open(os.path.join(GOLDEN, "qcx", "fused_brick.qcx")).read(), precision=pkg.C64,
                             keep_state=True)
    with state:
        a = state.amplitudes().astype(np.complex128)
        ref = arrays["fused_brick"]
        assert np.abs(a - ref).max() <= 2e-5
        assert abs(np.vdot(ref, a)) ** 2 / np.vdot(a, a).real >= 1 - 1e-9


def test_command_line_drop_in(pkg, expected):
    exp, _ = expected
    exe = os.path.join(ROOT, "riken-braket_b200", "bin", "rbk-bra")
    for name in ("hadamards8", "shor_program", "exit_program"):
        path = os.path.join(GOLDEN, "qcx", name + ".qcx")
        r = subprocess.run([exe, "--file", path, "--no-timing", "--threads", "4"], capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr
        same_output(r.stdout, exp[name]["output"])
    r = subprocess.run([exe, "--no-timing"], input="QUBITS 2\nH 0\nCNOT 0 1\nBOGUS 1\n", capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 1 and "line 4" in r.stderr


def test_seed_option_changes_the_state_generator(pkg):
    text = "QUBITS 6\n" + "".join("H %d\n" % q for q in range(6)) + "GENERATE EVENTS 30 -1\n"
    a, _ = pkg.qcx.run(text, seed=1)
    b, _ = pkg.qcx.run(text, seed=2)
    c, _ = pkg.qcx.run(text, seed=1)
    assert a == c and a != b


def test_waits_that_never_resolve_are_an_error(pkg):
    """bra's scheduler would loop forever here (circuit 1 finishes without the
    INNERPROD circuit 0 waits for); the engine reports it instead."""
    text = "CIRCUITS 2\nQUBITS 3\nH 0\nINNERPROD 1\nBEGIN CIRCUIT 1\nH 1\nEND CIRCUIT\n"
    with pytest.raises(pkg.RbkError) as e:
        pkg.qcx.run(text)
    assert e.value.code == 6


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n", [5, 12, 17])
def test_inner_product_pauli_vs_reference(pkg, n, precision):
    """<b| P |a> through rbk_inner_product_pauli against ket::runtime::ranges::inner_product
    with bra's observable (oracle KetRef.inner_product_on); sums of terms by linearity."""
    import oracle
    rng = np.random.default_rng(n + 10 * precision)
    va = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    vb = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    va /= np.linalg.norm(va)
    vb /= np.linalg.norm(vb)
    ra, rb = oracle.KetRef(n), oracle.KetRef(n)
    ra.set_amplitudes(va)
    rb.set_amplitudes(vb)
    a, b = pkg.State(n, precision), pkg.State(n, precision)
    a.upload(va)
    b.upload(vb)
    # queued gates on both (a SWAP relabels a's layout only) before the overlap
    a.apply([("H", (1,), ()), ("SWAP", (0, n - 1), ()), ("CNOT", (2, 3), ())])
    b.apply([("U3", (n - 2,), (0.3, 0.7, -1.1))])
    ra.apply([("H", (1,), ()), ("SWAP", (0, n - 1), ()), ("CNOT", (2, 3), ())])
    rb.apply([("U3", (n - 2,), (0.3, 0.7, -1.1))])
    tol = 1e-12 if precision == 0 else 1e-5
    total_ref, terms = 0j, []
    for k in range(4):
        m = int(rng.integers(1, min(n, 6) + 1))
        qubits = [int(q) for q in rng.choice(n, size=m, replace=False)]
        pauli = "".join(rng.choice(list("IXYZ"), size=m))
        want = ra.inner_product_on(rb, pauli, qubits)
        full = ["I"] * n
        for q, ch in zip(qubits, pauli):
            full[q] = ch
        full = "".join(full)
        got = a.inner_product_pauli(b, [(full, 1.0)])
        assert abs(got - want) <= tol, (pauli, qubits)
        assert abs(a.fidelity_pauli(b, [(full, 1.0)]) - abs(want) ** 2) <= tol
        c = complex(rng.standard_normal(), rng.standard_normal())
        terms.append((full, c))
        total_ref += c * want
    assert abs(a.inner_product_pauli(b, terms) - total_ref) <= 4 * tol
    a.close()
    b.close()


def test_pauliss_hamiltonian_energy_full_precision(pkg):
    """Config 4's Hamiltonian written as a .qcx program with PAULISS variables
    (tests/golden/qcx/pauliss_hamiltonian.qcx): the ansatz state the program
    leaves behind has the energy that EXPECTATION H printed, and it equals
    rbk_expectation_pauli on that state and the reference's own ket code
    (bra's EXPECTATION term by term, ketref_expectation_on) to 1e-12."""
    import oracle
    import bra_ref

    text = open(os.path.join(GOLDEN, "qcx", "pauliss_hamiltonian.qcx")).read()
    out, state = pkg.qcx.parse(text).run(keep_state=True)
    n = 10
    energy_engine = state.expectation(pkg.circuits.ansatz_hamiltonian(n))
    state.close()
    # The reference: the program's gates on ket as bra dispatches them, H term by term.
    _, _, code = bra_ref.parse(text)
    r = oracle.KetRef(n)
    for ins in code:
        if ins["op"] == bra_ref.OP["GATE"]:
            r.gate(ins["kind"], ins["targets"], ins["controls"], ins["params"])
    energy_ref = sum(r.expectation_on("ZZ", [i, (i + 1) % n]) for i in range(n))
    energy_ref += 0.5 * sum(r.expectation_on("X", [i]) for i in range(n))
    printed = complex(*(float(x) for x in out.splitlines()[0].strip("()").split(",")))
    assert abs(energy_engine - energy_ref) <= TOL64
    assert abs(printed - energy_ref) <= 1e-5 * max(1.0, abs(energy_ref))


@pytest.mark.parametrize("body,message", [
    ("VAR H PAULISS\nLET H += :PAULIS:ZZ\n", "wrong length"),            # a new variable has zero qubits
    ("VAR H PAULISS\nLET H := :PAULIS:ZZ\nEXPECTATION H 0 1 2\n", "qubits"),
    ("LET G := :PAULIS:ZZ\n", "not a PAULISS variable"),
    ("VAR H PAULISS\nVAR H PAULISS\n", "declared twice"),
    ("VAR H PAULISS 2\nLET H:2 := :PAULIS:Z\n", "out of range"),
    ("VAR H PAULISS\nLET H := :PAULIS:Z\nLET H *= 2.0\n", "complex value"),
])
def test_pauliss_errors_name_the_line(pkg, body, message):
    text = "QUBITS 3\nH 0\n" + body
    with pytest.raises(pkg.RbkError) as e:
        pkg.qcx.parse(text).run()
    assert message in str(e.value) and "line" in str(e.value)
