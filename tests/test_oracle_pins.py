"""Pins the oracle (CPU, no GPU).

The C restatement (oracle/rbk_oracle.c) is checked against fixtures that the
reference's own ket / bra code produced (tests/golden/, made by
tests/golden/make_golden.py from oracle/_ref), and -- where oracle/_ref is
built -- against the reference directly on fresh seeded circuits, including
bra's fused path.  Gate results must agree to the last bit; reductions to 1e-14.
"""
import os

import numpy as np
import pytest

import oracle
from conftest import ROOT, as_ops

REF_BUILT = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libketref.so"))
CIRCUITS = ["random6", "random9", "brick10_fused5", "brick12", "qft_brick8", "ansatz8", "hadamards08"]


def test_single_gates_match_reference_fixtures(golden):
    meta, arr = golden
    n = meta["single"]["n"]
    for i, op in enumerate(as_ops(meta["single"]["ops"])):
        o = oracle.COracle(n)
        o.set_amplitudes(arr["single_init"])
        o.apply([op])
        np.testing.assert_array_equal(o.amplitudes(), arr["single_out"][i], err_msg=str(op))


@pytest.mark.parametrize("name", CIRCUITS)
def test_circuits_match_reference_fixtures(golden, pkg, name):
    meta, arr = golden
    n = meta[name]["n"]
    o = oracle.COracle(n)
    o.apply(as_ops(meta[name]["ops"]))
    np.testing.assert_array_equal(o.amplitudes(), arr[f"{name}_amps"])
    np.testing.assert_allclose(o.spins(), arr[f"{name}_spins"], rtol=0, atol=1e-14)
    e = o.expectation(pkg.circuits.ansatz_hamiltonian(n))
    assert abs(e - arr[f"{name}_energy"][0]) < 1e-13


def test_hadamards08_known_answer(golden):
    # bra/qcx/hadamards08.qcx: 8 H gates on |0...0>, every amplitude 1/16, every <Z> = 0.
    _, arr = golden
    np.testing.assert_allclose(arr["hadamards08_amps"], np.full(256, 1 / 16), rtol=0, atol=1e-15)
    np.testing.assert_allclose(arr["hadamards08_spins"][:, 2], 0, atol=1e-15)


def test_brick20_matches_reference_fixture(golden, pkg):
    meta, arr = golden
    o = oracle.COracle(20)
    o.apply(pkg.circuits.brick(20, 10, seed=1))
    a = o.amplitudes()
    np.testing.assert_array_equal(a[arr["brick20_idx"]], arr["brick20_amps_sample"])
    np.testing.assert_allclose((np.abs(a) ** 2).reshape(1024, -1).sum(axis=1), arr["brick20_block_probs"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(o.spins(), arr["brick20_spins"], rtol=0, atol=1e-13)


@pytest.mark.skipif(not REF_BUILT, reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("seed", [21, 22, 23])
def test_restatement_equals_reference_on_fresh_circuits(pkg, seed):
    C = pkg.circuits
    n = 7
    ops = C.random_circuit(n, 250, seed=seed)
    # wrap a stretch in a fusion block so bra's fused replay is exercised
    ops = ops[:50] + [("BEGIN FUSION", (), ())] + [op for op in ops[50:90] if op[0] != "SWAP"] + \
        [("END FUSION", (), ())] + ops[90:]
    r = oracle.KetRef(n)
    r.apply(ops)
    o = oracle.COracle(n)
    o.apply(ops)
    np.testing.assert_array_equal(o.amplitudes(), r.amplitudes())
    np.testing.assert_allclose(o.spins(), r.spins(), rtol=0, atol=1e-14)
    terms = [("XYZIIII", 0.5), ("YYYYYYY", 1j), ("ZIIIIIZ", -1.0)]
    assert abs(o.expectation(terms) - r.expectation(terms)) < 1e-14
    r2 = oracle.KetRef(n, initial_index=5)
    o2 = oracle.COracle(n, initial_index=5)
    assert abs(o.inner_product(o2) - r.inner_product(r2)) < 1e-14


@pytest.mark.skipif(not REF_BUILT, reason="oracle/_ref not built (needs the reference sources)")
def test_reference_fused_brick_equals_unfused(pkg):
    C = pkg.circuits
    a = oracle.KetRef(10)
    a.apply(C.brick(10, 4, seed=9, fuse_k=5))
    b = oracle.COracle(10)
    b.apply(C.brick(10, 4, seed=9))
    np.testing.assert_allclose(a.amplitudes(), b.amplitudes(), rtol=0, atol=1e-14)


def test_sampling_restatement_matches_reference_fixtures(golden):
    """MT19937-64 + uniform_real_distribution + upper_bound over the prefix of
    |a|^2 (generate_events.hpp), projective_measurement.hpp and measure.hpp:
    indices and outcomes equal, collapsed amplitudes bit-equal."""
    meta, arr = golden
    n = meta["random9"]["n"]
    ops = as_ops(meta["random9"]["ops"])

    def fresh():
        o = oracle.COracle(n)
        o.apply(ops)
        return o

    assert np.array_equal(fresh().generate_events(2000, 5), arr["random9_events_seeded"])
    assert np.array_equal(fresh().generate_events(2000), arr["random9_events_state_rng"])
    o = fresh()
    o.seed(23)
    outs = [o.projective_measurement(int(q)) for q in arr["random9_projective_qubits"]]
    assert outs == list(arr["random9_projective_outcomes"])
    assert np.array_equal(o.amplitudes(), arr["random9_projective_amps"])
    assert o.measure() == arr["random9_measure"][0]


@pytest.mark.skipif(not REF_BUILT, reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("n", [7, 12])
def test_sampling_restatement_equals_reference_on_fresh_states(pkg, n):
    ops = pkg.circuits.random_circuit(n, 250, seed=n)
    r, o = oracle.KetRef(n), oracle.COracle(n)
    r.apply(ops)
    o.apply(ops)
    r.seed(n)
    o.seed(n)
    for q in range(n):
        assert r.projective_measurement(q) == o.projective_measurement(q)
    assert np.array_equal(r.amplitudes(), o.amplitudes())
    r, o = oracle.KetRef(n), oracle.COracle(n)
    r.apply(ops)
    o.apply(ops)
    assert np.array_equal(o.generate_events(5000, 77), r.generate_events(5000, 77))
    r, o = oracle.KetRef(n), oracle.COracle(n)  # the reference left prefix sums in its buffer
    r.apply(ops)
    o.apply(ops)
    assert r.measure() == o.measure()
    assert np.array_equal(r.amplitudes(), o.amplitudes())


@pytest.mark.parametrize("prog", ["runtime_gate_numerical", "fused_runtime_gate_numerical", "runtime_observable_numerical"])
def test_reference_own_tests_pass_with_shim(prog):
    """The reference's ket/test/*.cpp, compiled unchanged against the Boost stand-ins (riken-braket_b200/bra/shim)."""
    import subprocess
    path = os.path.join(ROOT, "oracle", "_ref", prog)
    if not os.path.exists(path):
        pytest.skip("reference tests not built (needs the reference sources)")
    r = subprocess.run([path], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "passed" in r.stdout
