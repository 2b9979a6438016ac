"""The .qcx front end on the CPU: the engine's C++ parser (include/rbk_qcx.h)
against the independent Python restatement in oracle/bra_ref.py, bra's
error behaviour, and the reference-run expectations the GPU tests use."""
import glob
import json
import os

import numpy as np
import pytest

import bra_ref
import oracle
from conftest import REFERENCE, ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")
PROGRAMS = sorted(glob.glob(os.path.join(GOLDEN, "qcx", "*.qcx")))
REF_BUILT = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libketref.so"))
REF_SAMPLES = os.path.join(REFERENCE, "bra", "qcx")
FIELDS = ("op", "kind", "line", "circuit", "targets", "controls", "params", "text")


def same_program(cpp, py):
    assert len(cpp) == len(py)
    for a, b in zip(cpp, py):
        for k in FIELDS:
            assert a[k] == b[k], (k, a, b)
        if a["op"] == bra_ref.OP["AMPLITUDES"]:
            assert a["values"] == b["values"][:40]
        if a["op"] in (bra_ref.OP["INNERPROD"], bra_ref.OP["FIDELITY"]):
            assert a["ints"][0] == b["ints"][0]


@pytest.mark.parametrize("path", PROGRAMS, ids=os.path.basename)
def test_cpp_parser_equals_python_restatement(pkg, path):
    text = open(path).read()
    prog = pkg.qcx.parse(text)
    n, init, code, circuits = bra_ref.parse_program(text)
    assert prog.num_qubits == n and prog.initial_state == init and prog.num_circuits == circuits
    same_program(prog.instructions(), code)


@pytest.mark.skipif(not os.path.isdir(REF_SAMPLES), reason="reference sample programs not present")
@pytest.mark.parametrize("name", ["adder6x2", "toffoli12", "shor12", "hadamards08"])
def test_reference_sample_programs_parse_identically(pkg, name):
    text = open(os.path.join(REF_SAMPLES, name + ".qcx")).read()
    n, _, code = bra_ref.parse(text)
    same_program(pkg.qcx.parse(text).instructions(), code)


def test_every_gate_program_covers_the_gate_set(pkg):
    kinds = {i["kind"] for i in pkg.qcx.parse(open(os.path.join(GOLDEN, "qcx", "every_gate.qcx")).read()).instructions()}
    assert set(range(1, 34)) <= kinds


@pytest.mark.parametrize("text,code,where", [
    ("QUBITS 3\nH 0\nFOO 1\n", 1, "line 3"),
    ("QUBITS 3\nH 3\n", 1, "line 2"),
    ("QUBITS 3\nCNOT 0\n", 1, "line 2"),
    ("QUBITS 3\nCNOT 1 1\n", 1, "line 2"),
    ("H 0\n", 1, "line 1"),
    ("QUBITS 3\nU3 0 1.0 2.0 x\n", 5, "line 2"),
    ("QUBITS 3\nVAR A INT\n", 5, "line 2"),
    ("CIRCUITS 2\nQUBITS 3\nBEGIN CIRCUIT 2\n", 1, "line 3"),
    ("CIRCUITS 2\nQUBITS 3\nBEGIN CIRCUIT 1\nBEGIN CIRCUIT 0\n", 1, "line 4"),
    ("QUBITS 3\nEND CIRCUIT\n", 1, "line 2"),
    ("QUBITS 3\nINNERPROD 1\n", 1, "line 2"),
    ("CIRCUITS 2\nQUBITS 3\nFIDELITY 1 :PAULIS:ZZ 0\n", 1, "line 3"),
    ("CIRCUITS 2\nQUBITS 3\nINNERPROD ALL :REAL:1 0 1\n", 5, "line 3"),
    ("QUBITS 3\nVAR H PAULISS\nLET H ** :PAULIS:Z\n", 1, "line 3"),
    ("QUBITS 3\nVAR 1H PAULISS\n", 1, "line 2"),
    ("QUBITS 3\nVAR H PAULISS 0\n", 1, "line 2"),
    ("QUBITS 3\nEXPECTATION :PAULIS:ZQ 0 1\n", 1, "line 2"),
    ("QUBITS 3\nDEPOLARIZING CHANNEL P_X=0.1\n", 5, "line 2"),
    ("QUBITS 3\nEXPECTATION :PAULIS:ZZ 0\n", 1, "line 2"),
    ("", 1, "QUBITS"),
])
def test_parse_errors_name_the_line(pkg, text, code, where):
    with pytest.raises(pkg.RbkError) as e:
        pkg.qcx.parse(text)
    assert e.value.code == code and where in str(e.value)


def test_comments_case_and_stops(pkg):
    prog = pkg.qcx.parse("! header\nqubits 4 ! four\n  h 0\ncnot 0 1\nExit\nH 9 garbage\n")
    ins = prog.instructions()
    assert [i["op"] for i in ins] == [1, 1, 7]  # EXIT ends the program text (bra stops reading)
    assert ins[1]["controls"] == [0] and ins[1]["targets"] == [1]
    ins = pkg.qcx.parse("QUBITS 3\nGENERATE EVENTS 5 -1\nH 0\n").instructions()
    assert len(ins) == 1 and ins[0]["ints"] == [5, -1]


def test_circuit_blocks_and_partners(pkg):
    text = ("CIRCUITS 3\nQUBITS 4\nH 0\nINNERPROD 0\nBEGIN CIRCUIT 2\nX 1\nFIDELITY ALL\nINNERPROD 2\n"
            "INNERPROD 0 :PAULIS:XZ 3 1\nEND CIRCUIT\nINNERPROD foo\nFIDELITY 2\n")
    prog = pkg.qcx.parse(text)
    ins = prog.instructions()
    assert prog.num_circuits == 3
    assert [i["circuit"] for i in ins] == [0, 0, 2, 2, 2, 2, 0, 0]
    # own index and a column that is neither a number nor ALL: nothing to wait for
    assert [i["ints"][0] for i in ins if i["op"] in (12, 13)] == [-2, -1, -2, 0, -2, 2]
    assert ins[5]["text"] == "XZ" and ins[5]["targets"] == [3, 1]


def test_run_without_gpu_is_a_cuda_error(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.RbkError) as e:
        pkg.qcx.run("QUBITS 2\nH 0\nDO MEASUREMENT\n")
    assert e.value.code == 2


@pytest.mark.skipif(not REF_BUILT, reason="oracle/_ref not built (needs the reference sources)")
def test_expected_outputs_reproduce_from_the_reference():
    expected = json.load(open(os.path.join(GOLDEN, "qcx_expected.json")))
    arrays = np.load(os.path.join(GOLDEN, "qcx_golden.npz"))
    for path in PROGRAMS:
        name = os.path.basename(path)[:-4]
        out, amps, _ = bra_ref.run(open(path).read())
        assert out == expected[name]["output"], name
        if expected[name]["amplitudes"]:
            assert np.array_equal(amps, arrays[name]), name


@pytest.mark.skipif(not REF_BUILT, reason="oracle/_ref not built (needs the reference sources)")
def test_hadamards_known_answer():
    """Every amplitude of H on 8 qubits is 1/16 (the reference's hadamards08 sample)."""
    _, amps, _ = bra_ref.run(open(os.path.join(GOLDEN, "qcx", "hadamards8.qcx")).read())
    assert np.allclose(amps, 1.0 / 16.0, atol=1e-15, rtol=0)
