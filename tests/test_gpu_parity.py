"""GPU parity: the CUDA path (through the C ABI of librbk.so) against the
oracle, on the same seeded inputs.  FP64 (c128) results must agree to 1e-12
max absolute amplitude error (the bar of the reference's own tests,
ket/test/runtime_gate_numerical.cpp:80-86); FP32 (c64) to 2e-5."""
import numpy as np
import pytest

import oracle
from conftest import as_ops

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return a / np.linalg.norm(a)


def run_both(pkg, n, ops, init=None, precision=0, deferred=True, budget=0):
    s = pkg.State(n, precision)
    s.set_deferred(deferred)
    if budget:
        s.set_pass_budget(budget)
    o = oracle.COracle(n)
    if init is not None:
        s.upload(init)
        o.set_amplitudes(init)
    s.apply(ops)
    o.apply(ops)
    return s, o


def test_single_gates_vs_reference_fixtures(pkg, golden):
    """Every hot-path gate alone on the 4-qubit state of the reference's tests
    (per-gate kernel path: the state is smaller than one tile)."""
    meta, arr = golden
    n = meta["single"]["n"]
    for i, op in enumerate(as_ops(meta["single"]["ops"])):
        s = pkg.State(n)
        s.upload(arr["single_init"])
        s.apply([op])
        got = s.amplitudes()
        assert np.abs(got - arr["single_out"][i]).max() <= TOL64, op
        s.close()


@pytest.mark.parametrize("name", ["random6", "random9", "brick10_fused5", "brick12", "qft_brick8", "ansatz8", "hadamards08"])
def test_circuits_vs_reference_fixtures(pkg, golden, name):
    meta, arr = golden
    n = meta[name]["n"]
    with pkg.State(n) as s:
        s.apply(as_ops(meta[name]["ops"]))
        assert np.abs(s.amplitudes() - arr[f"{name}_amps"]).max() <= TOL64
        assert np.abs(s.spins() - arr[f"{name}_spins"]).max() <= TOL64
        e = s.expectation(pkg.circuits.ansatz_hamiltonian(n))
        assert abs(e - arr[f"{name}_energy"][0]) <= TOL64


@pytest.mark.parametrize("n", [12, 13, 15, 17])
@pytest.mark.parametrize("seed", [1, 2])
def test_random_circuits_fused_tile_path(pkg, n, seed):
    """Random mixes of every gate kind on states of one tile and more, so
    targets and controls land in registers, thread bits and outside the tile."""
    ops = pkg.circuits.random_circuit(n, 400, seed=seed)
    s, o = run_both(pkg, n, ops, init=random_state(n, seed))
    assert np.abs(s.amplitudes() - o.amplitudes()).max() <= TOL64
    st = s.stats()
    assert st["passes"] >= 1 and st["gate_launches"] == 0


@pytest.mark.parametrize("n", [13, 16])
def test_controlled_gates_every_position(pkg, n):
    """Controlled 2x2 gates with every target and a control on each side."""
    rng = np.random.default_rng(n)
    ops = []
    for t in range(n):
        for c in (t - 1, t + 1, n - 1 - t):
            if 0 <= c < n and c != t:
                a = [float(x) for x in rng.uniform(0, 6.28, 3)]
                ops.append(("CNOT", (c, t), ()))
                ops.append(("CZ", (c, t), ()))
                ops.append(("U", (c, t), (int(rng.integers(1, n)),)))
        ops.append(("U3", (t,), tuple(float(x) for x in rng.uniform(0, 6.28, 3))))
    s, o = run_both(pkg, n, ops, init=random_state(n, 3))
    assert np.abs(s.amplitudes() - o.amplitudes()).max() <= TOL64
    # multi-controlled gates through the C ABI directly
    s2 = pkg.State(n)
    s2.upload(random_state(n, 4))
    ref = random_state(n, 4)
    s2.u3(0.3, 1.1, 2.2, 5, controls=(0, n - 1, 9))
    s2.pauli_x(n - 2, controls=(1, 6))
    s2.hadamard(0, controls=(n - 1,))
    s2.pauli_y(3, controls=(11,))
    s2.synchronize()
    got = s2.amplitudes()

    def ctrl_apply(a, m, t, cs):
        a = a.copy()
        idx = np.arange(1 << n)
        sel = (idx >> t) & 1 == 0
        for c in cs:
            sel &= (idx >> c) & 1 == 1
        i0 = idx[sel]
        i1 = i0 | (1 << t)
        a0, a1 = a[i0].copy(), a[i1].copy()
        a[i0] = m[0, 0] * a0 + m[0, 1] * a1
        a[i1] = m[1, 0] * a0 + m[1, 1] * a1
        return a

    th, ph, la = 0.3, 1.1, 2.2
    u3 = np.array([[np.cos(th / 2), -np.exp(1j * la) * np.sin(th / 2)],
                   [np.exp(1j * ph) * np.sin(th / 2), np.exp(1j * (ph + la)) * np.cos(th / 2)]])
    ref = ctrl_apply(ref, u3, 5, (0, n - 1, 9))
    ref = ctrl_apply(ref, np.array([[0, 1], [1, 0]]), n - 2, (1, 6))
    ref = ctrl_apply(ref, np.array([[1, 1], [1, -1]]) / np.sqrt(2), 0, (n - 1,))
    ref = ctrl_apply(ref, np.array([[0, -1j], [1j, 0]]), 3, (11,))
    assert np.abs(got - ref).max() <= TOL64


def test_brick20_config1_vs_reference_fixture(pkg, golden):
    """The 20-qubit brick (H layer + 10 layers of U3 and CNOT) against the
    reference's outputs: sampled amplitudes, block probabilities, spins."""
    _, arr = golden
    with pkg.State(20) as s:
        s.apply(pkg.circuits.brick(20, 10, seed=1))
        a = s.amplitudes()
        assert np.abs(a[arr["brick20_idx"]] - arr["brick20_amps_sample"]).max() <= TOL64
        probs = s.probabilities()
        assert np.abs(probs.reshape(1024, -1).sum(axis=1) - arr["brick20_block_probs"]).max() <= TOL64
        assert np.abs(s.spins() - arr["brick20_spins"]).max() <= TOL64
        assert np.abs(probs - np.abs(a) ** 2).max() <= 1e-15


def test_brick20_full_state_vs_oracle(pkg):
    n, ops = 20, pkg.circuits.brick(20, 10, seed=1, fuse_k=5)
    s, o = run_both(pkg, n, ops)
    assert np.abs(s.amplitudes() - o.amplitudes()).max() <= TOL64


@pytest.mark.parametrize("budget", [1, 4, 40])
def test_pass_budget_and_immediate_mode_agree(pkg, budget):
    n = 16
    ops = pkg.circuits.brick(n, 6, seed=5) + pkg.circuits.random_circuit(n, 200, seed=6)
    init = random_state(n, 7)
    s, o = run_both(pkg, n, ops, init=init, budget=budget)
    want = o.amplitudes()
    assert np.abs(s.amplitudes() - want).max() <= TOL64
    s2, _ = run_both(pkg, n, ops, init=init, deferred=False)
    assert np.abs(s2.amplitudes() - want).max() <= TOL64
    assert s2.stats()["passes"] >= len([op for op in ops if op[0] != "SWAP"])


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("shape", [0, 2, 3])
def test_every_tile_shape_vs_oracle(pkg, shape, precision):
    """Each tile shape (3: the persistent CTAs that copy their next tile with
    cp.async) on a brick plus random gates, at sizes from one tile to many
    tiles per CTA, in both precisions."""
    tol = TOL64 if precision == 0 else TOL32
    for n in (13, 17, 21):
        ops = pkg.circuits.brick(n, 4, seed=n + shape) + pkg.circuits.random_circuit(n, 150, seed=n + 10 * shape)
        init = random_state(n, n + shape)
        s = pkg.State(n, precision)
        s.set_tile_shape(shape)
        s.upload(init)
        o = oracle.COracle(n)
        o.set_amplitudes(init)
        s.apply(ops)
        o.apply(ops)
        assert np.abs(s.amplitudes().astype(np.complex128) - o.amplitudes()).max() <= tol, (n, shape, precision)
        assert s.stats()["passes"] >= 1
        s.close()


def test_tile_shape_1_is_rejected(pkg):
    with pkg.State(13) as s:
        with pytest.raises(pkg.RbkError):
            s.set_tile_shape(1)


def test_layout_map_swaps_and_canonicalize(pkg):
    n = 18
    rng = np.random.default_rng(8)
    ops = []
    for _ in range(60):
        a, b = (int(x) for x in rng.permutation(n)[:2])
        ops.append(("SWAP", (a, b), ()))
        ops.append(("U3", (int(rng.integers(n)),), tuple(float(x) for x in rng.uniform(0, 6.28, 3))))
    s, o = run_both(pkg, n, ops, init=random_state(n, 9))
    s.flush()
    perm = s.permutation()
    assert sorted(perm) == list(range(n))
    # observables read through the layout map without moving data
    assert np.abs(s.spins() - o.spins()).max() <= TOL64
    assert np.abs(s.amplitudes() - o.amplitudes()).max() <= TOL64
    assert s.permutation() == list(range(n))
    # controlled swap is three exact controlled-X permutations
    before = s.amplitudes()
    s.swap(2, 15, controls=(7,))
    idx = np.arange(1 << n)
    b2, b15 = (idx >> 2) & 1, (idx >> 15) & 1
    src = np.where(((idx >> 7) & 1) == 1, idx ^ ((b2 ^ b15) * ((1 << 2) | (1 << 15))), idx)
    np.testing.assert_array_equal(s.amplitudes(), before[src])


def _permute_bits(perm, idx):
    """Index whose bit perm[q] is bit q of idx (ket::mpi::permutate_bits)."""
    out = np.zeros_like(idx)
    for q, p in enumerate(perm):
        out |= ((idx >> q) & 1) << p
    return out


@pytest.mark.parametrize("n,precision", [(9, 0), (18, 0), (18, 1)])
def test_set_layout_and_set_permutation(pkg, n, precision):
    """rbk_state_set_layout moves the data (the logical state stays the
    oracle's); rbk_state_set_permutation relabels without moving it, so the
    logical state becomes the physical data read under the new map."""
    tol = TOL64 if precision == 0 else 2e-5
    ops = pkg.circuits.random_circuit(n, 120, seed=31 + n)
    s = pkg.State(n, precision)
    s.upload(random_state(n, 5).astype(s.dtype))
    s.apply(ops)
    o = oracle.COracle(n)
    o.set_amplitudes(random_state(n, 5).astype(s.dtype).astype(np.complex128))
    o.apply(ops)
    want = o.amplitudes()
    rng = np.random.default_rng(n)
    target = [int(x) for x in rng.permutation(n)]
    s.set_layout(target)
    assert s.permutation() == target
    idx = np.arange(1 << n, dtype=np.int64)
    phys = np.empty_like(want)
    phys[_permute_bits(target, idx)] = want                    # the device memory now
    # Declare the identity map: the logical state becomes the memory as it lies.
    # (Reads bring the memory into logical order, so nothing is read before.)
    s.set_permutation(list(range(n)))
    assert np.abs(s.amplitudes() - phys).max() <= tol
    # The memory is in identity order now; declaring `target` gives back the circuit's state.
    s.set_permutation(target)
    assert np.abs(s.amplitudes() - want).max() <= tol
    # set_layout keeps the logical state.
    s.set_layout(target[::-1])
    assert s.permutation() == target[::-1]
    assert np.abs(s.amplitudes() - want).max() <= tol
    with pytest.raises(pkg.RbkError):
        s.set_permutation([0] * n)
    s.close()


@pytest.mark.parametrize("n", [10, 14, 19])
def test_observables_vs_oracle(pkg, n):
    ops = pkg.circuits.random_circuit(n, 150, seed=n)
    s, o = run_both(pkg, n, ops, init=random_state(n, n + 1))
    assert abs(s.norm2() - 1.0) <= TOL64
    assert np.abs(s.spins() - o.spins()).max() <= TOL64
    terms = pkg.circuits.ansatz_hamiltonian(n) + [("XYZ" + "I" * (n - 3), 0.3 + 0.1j), ("Y" * n, 1.0),
                                                  ("I" * (n - 2) + "YX", -0.5j), ("Z" * n, 2.0)]
    assert abs(s.expectation(terms) - o.expectation(terms)) <= TOL64
    t = pkg.State(n)
    t.upload(random_state(n, 99))
    o2 = oracle.COracle(n)
    o2.set_amplitudes(random_state(n, 99))
    assert abs(s.inner_product(t) - o.inner_product(o2)) <= TOL64
    assert abs(s.fidelity(t) - abs(o.inner_product(o2)) ** 2) <= TOL64
    p = s.probabilities(offset=3, count=(1 << n) - 5)
    assert np.abs(p - o.probabilities()[3:-2]).max() <= 1e-15


@pytest.mark.parametrize("n", [13, 16, 20])
def test_c64_path_vs_fp64_oracle(pkg, n):
    ops = pkg.circuits.brick(n, 5, seed=n) + pkg.circuits.random_circuit(n, 120, seed=n)
    s, o = run_both(pkg, n, ops, precision=pkg.C64)
    got = s.amplitudes().astype(np.complex128)
    want = o.amplitudes()
    assert np.abs(got - want).max() <= TOL32
    # FP32-rounded gate matrices are unitary only to ~1e-7, so the norm drifts;
    # fidelity is taken against the normalised result.
    norm = np.vdot(got, got).real
    assert abs(norm - 1.0) < 1e-4
    fidelity = abs(np.vdot(want, got)) ** 2 / norm
    assert fidelity > 1 - 1e-6
    assert np.abs(s.spins() - o.spins()).max() <= 1e-5


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n", [3, 11, 12, 17, 23])
def test_spins_all_layouts_vs_oracle(pkg, n, precision):
    """Every qubit's spins from the tiled layouts (one read of the state per
    layout), after queued SWAPs moved logical qubits around the physical bits."""
    ops = pkg.circuits.random_circuit(n, 80, seed=n + 3) + [("SWAP", (0, n - 1), ()), ("SWAP", (1, n // 2 + 1), ())]
    init = random_state(n, n + 7)
    s, o = run_both(pkg, n, ops, init=init, precision=precision)
    tol = TOL64 if precision == 0 else 2e-6
    assert np.abs(s.spins() - o.spins()).max() <= tol


def test_errors_are_status_codes(pkg):
    s = pkg.State(14)
    with pytest.raises(pkg.RbkError) as e:
        s.hadamard(14)
    assert e.value.code == 1
    with pytest.raises(pkg.RbkError) as e:
        s.pauli_x(3, controls=(3,))
    assert e.value.code == 1
    with pytest.raises(pkg.RbkError) as e:
        s.pauli_z(2, 2)
    assert e.value.code == 1
    with pytest.raises(pkg.RbkError) as e:
        s.end_fusion()
    assert e.value.code == 6
    s.begin_fusion()
    with pytest.raises(pkg.RbkError) as e:
        s.begin_fusion()
    assert e.value.code == 6
    with pytest.raises(pkg.RbkError) as e:
        s.controlled_phase_shift_k(15, 0, 1)
    assert e.value.code == 1
    with pytest.raises(pkg.RbkError):
        pkg.State(34, pkg.C128)
    with pytest.raises(pkg.RbkError):
        s.amplitudes(offset=1 << 14, count=1)
    # the state is still usable after rejected calls
    s.end_fusion()
    s.hadamard(0)
    assert abs(s.norm2() - 1.0) < 1e-14


def test_observables_right_after_queued_swaps(pkg):
    """Reads issued straight after gates that move qubits (SWAPs, relabelling)
    see the layout those gates leave behind."""
    n = 16
    ops = pkg.circuits.random_circuit(n, 200, seed=5)
    terms = pkg.circuits.ansatz_hamiltonian(n) + [("XYZ" + "I" * (n - 3), 0.3 + 0.1j)]
    o = oracle.COracle(n)
    o.apply(ops)
    s = pkg.State(n)
    s.apply(ops)
    assert abs(s.expectation(terms) - o.expectation(terms)) <= TOL64
    a, b = pkg.State(n), pkg.State(n)
    a.apply(ops)
    b.apply(ops[:120])
    ob = oracle.COracle(n)
    ob.apply(ops[:120])
    assert abs(a.inner_product(b) - o.inner_product(ob)) <= TOL64


def layer_circuit(n, seed):
    """Runs of uncontrolled single-qubit gates on subsets of a few neighbouring
    qubits, in every matrix form the layer blocks take (H: real; U3: m00 real;
    H then U3 on one qubit, which the planner merges: general), separated by
    CNOTs inside the window, so that register phases hold layers over every
    mask of register bits and mixed forms."""
    rng = np.random.default_rng(seed)
    ops = []
    for _ in range(40):
        lo = int(rng.integers(0, n - 6))
        window = list(range(lo, lo + 6))
        subset = [q for q in window if rng.random() < 0.6] or [window[0]]
        for q in subset:
            form = int(rng.integers(3))
            angles = tuple(float(x) for x in rng.uniform(0.0, 2.0 * np.pi, size=3))
            if form == 0:
                ops.append(("H", (q,), ()))
            elif form == 1:
                ops.append(("U3", (q,), angles))
            else:
                ops += [("H", (q,), ()), ("U3", (q,), angles)]
        for _ in range(int(rng.integers(0, 3))):
            c, t = (int(x) for x in rng.permutation(window)[:2])
            ops.append(("CNOT", (c, t), ()))
    return ops


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("budget", [4, 8, 0])
def test_layer_blocks_every_mask_and_form(pkg, precision, budget):
    n = 15
    tol = TOL64 if precision == 0 else TOL32
    ops = layer_circuit(n, 100 + budget)
    init = random_state(n, 11)
    s, o = run_both(pkg, n, ops, init=init, precision=precision, budget=budget)
    assert np.abs(s.amplitudes().astype(np.complex128) - o.amplitudes()).max() <= tol
    s.close()


def phase_run_circuit(n, seed):
    """Long runs of phase gates (controlled phases U m j k, CZ, Z, U1) whose
    bits fall on register bits, thread bits and bits outside the tile, in every
    combination, between dense layers; every accumulator class of a phase run
    is exercised."""
    rng = np.random.default_rng(seed)
    ops = [("H", (q,), ()) for q in range(n)]
    for _ in range(6):
        for _ in range(60):
            a, b = (int(x) for x in rng.permutation(n)[:2])
            kind = int(rng.integers(4))
            if kind == 0:
                k = int(rng.integers(1, n + 1))
                ops.append(("U", (a, b), (k if rng.random() < 0.7 else -k,)))
            elif kind == 1:
                ops.append(("CZ", (a, b), ()))
            elif kind == 2:
                ops.append(("Z", (a,), ()))
            else:
                ops.append(("U1", (a,), (float(rng.uniform(0.0, 2.0 * np.pi)),)))
        for q in rng.permutation(n)[:5]:
            ops.append(("U3", (int(q),), tuple(float(x) for x in rng.uniform(0.0, 2.0 * np.pi, size=3))))
    return ops


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n", [13, 18])
def test_phase_runs_every_accumulator_class(pkg, precision, n):
    tol = TOL64 if precision == 0 else TOL32
    ops = phase_run_circuit(n, 200 + n)
    init = random_state(n, 12)
    s, o = run_both(pkg, n, ops, init=init, precision=precision)
    assert np.abs(s.amplitudes().astype(np.complex128) - o.amplitudes()).max() <= tol
    s.close()
