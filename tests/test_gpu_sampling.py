"""GPU sampling and measurement against the reference's fixtures and the oracle.

ket::generate_events (ket/include/ket/generate_events.hpp), ket::measure
(ket/include/ket/measure.hpp) and ket::gate::projective_measurement
(ket/include/ket/gate/projective_measurement.hpp) draw from std::mt19937_64
through uniform_real_distribution; the engine draws the same numbers on the
host, so event indices must be equal, not only equally distributed.  The one
source of disagreement is the prefix sum of |a|^2, which the device adds in
a different order: an event can move to a neighbouring index only when its
random number falls within rounding of a bin edge (probability ~1e-13 per
event at these sizes), so the tests demand equality."""
import numpy as np
import pytest

import oracle
from conftest import as_ops

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _random9(pkg, golden, precision=0):
    meta, arr = golden
    s = pkg.State(meta["random9"]["n"], precision)
    s.apply(as_ops(meta["random9"]["ops"]))
    return s, arr


def test_generate_events_seeded_vs_reference_fixture(pkg, golden):
    s, arr = _random9(pkg, golden)
    with s:
        before = s.amplitudes()
        ev = s.generate_events(2000, 5)
        assert np.array_equal(ev, arr["random9_events_seeded"])
        # the engine leaves the amplitudes alone (the reference overwrites them with prefix sums)
        assert np.array_equal(s.amplitudes(), before)


def test_generate_events_state_generator_vs_reference_fixture(pkg, golden):
    s, arr = _random9(pkg, golden)
    with s:
        assert np.array_equal(s.generate_events(2000), arr["random9_events_state_rng"])


def test_projective_measurements_and_measure_vs_reference_fixture(pkg, golden):
    s, arr = _random9(pkg, golden)
    with s:
        s.seed(23)
        outcomes = [s.projective_measurement(int(q)) for q in arr["random9_projective_qubits"]]
        assert outcomes == list(arr["random9_projective_outcomes"])
        assert np.abs(s.amplitudes() - arr["random9_projective_amps"]).max() <= TOL64
        assert s.measure() == arr["random9_measure"][0]
        a = s.amplitudes()
        assert a[arr["random9_measure"][0]] == 1 and np.count_nonzero(a) == 1


@pytest.mark.parametrize("n", [14, 18, 22])
def test_events_after_fused_passes_and_swaps_vs_oracle(pkg, n):
    """Deferred fused passes with SWAPs (layout map not identity) before sampling."""
    C = pkg.circuits
    ops = C.brick(n, 4, seed=n) + [("SWAP", (0, n - 1), ()), ("SWAP", (1, n // 2), ())] + C.random_circuit(n, 60, seed=n)
    s = pkg.State(n)
    s.apply(ops)
    o = oracle.COracle(n)
    o.apply(ops)
    with s:
        s.seed(n)
        o.seed(n)
        a = s.generate_events(10000)
        b = o.generate_events(10000)
        assert np.count_nonzero(a != b) == 0
        assert np.array_equal(s.generate_events(3000, 99), o.generate_events(3000, 99))
        outs = [(s.projective_measurement(q), o.projective_measurement(q)) for q in (n - 1, 0, n // 2)]
        assert all(x == y for x, y in outs), outs
        assert np.abs(s.amplitudes() - o.amplitudes()).max() <= TOL64
        assert abs(s.norm2() - 1.0) <= 1e-12


def test_c64_events_follow_the_same_distribution(pkg, golden):
    s64, _ = _random9(pkg, golden, precision=1)
    s128, _ = _random9(pkg, golden)
    with s64, s128:
        a = s64.generate_events(20000, 3)
        b = s128.generate_events(20000, 3)
        # same random numbers, bins differ by fp32 rounding of the amplitudes only
        assert np.count_nonzero(a != b) <= 20


def test_sampling_edge_cases(pkg):
    with pkg.State(6, initial_index=45) as s:
        assert s.generate_events(0).size == 0
        assert np.all(s.generate_events(100, 1) == 45)  # a basis state: every event is its index
        assert s.projective_measurement(0) == 1 and s.projective_measurement(1) == 0
        with pytest.raises(pkg.RbkError):
            s.projective_measurement(6)
        assert pkg.rbk.lib().rbk_generate_events(s.h, -1, 0, None) != 0
        s.hadamard(5)
        # |101101> -> (|001101> - |101101>)/sqrt2 after H on qubit 5 (bit 5 was set)
        ev = s.generate_events(4000, 2)
        assert set(np.unique(ev)) == {13, 45}
        assert 1800 < np.count_nonzero(ev == 13) < 2200
        assert s.measure() in (13, 45)
