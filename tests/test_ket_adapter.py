"""ket's template API on the device (include/rbk_ket.hpp).

The same ket program (tests/host/ket_adapter_check.cpp) runs with ket's
sequential policy on a std::vector -- ket's own code -- and with the b200
policy on an rbk::device_state; amplitudes and observables must agree to
1e-12 (complex<double>) / 2e-5 (complex<float>), and events, measurement
outcomes and projective-measurement outcomes drawn from equally seeded engines
must be the same (complex<double>).  The program is built by
`build()` into oracle/_ref where ket's headers are available.
"""
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARY = os.path.join(ROOT, "oracle", "_ref", "ket_adapter_check")
from conftest import REFERENCE  # noqa: E402

KET_INCLUDE = os.path.join(REFERENCE, "ket", "include")

_HEADER_ONLY_TU = r"""
#include <complex>
#include <random>
#include <vector>
#include <ket/qubit.hpp>
#include <ket/control.hpp>
#include "rbk_ket.hpp"
// Instantiates every overload family once for each precision.
template <typename Complex>
void every_gate(rbk::device_state<Complex>& s)
{
  namespace g = ket::gate::ranges;
  auto const p = ket::utility::policy::make_b200();
  using q_t = ket::qubit<std::uint64_t, unsigned>;
  q_t const a{0u}, b{1u}, d{2u};
  auto const c = ket::make_control(b);
  std::complex<double> const z{0.6, 0.8};
  g::hadamard(p, s, a, c); g::adj_hadamard(p, s, a);
  g::pauli_x(p, s, a, d, c); g::adj_pauli_x(p, s, a); g::not_(p, s, a, c); g::adj_not_(p, s, a);
  g::controlled_not(p, s, a, c); g::adj_controlled_not(p, s, a, c);
  g::toffoli(p, s, a, c, ket::make_control(d)); g::adj_toffoli(p, s, a, c, ket::make_control(d));
  g::pauli_y(p, s, a, c); g::adj_pauli_y(p, s, a, d);
  g::pauli_z(p, s, a, c); g::pauli_z(p, s, c, ket::make_control(a)); g::adj_pauli_z(p, s, a); g::adj_pauli_z(p, s, c);
  g::phase_shift_coeff(p, s, z, a, c); g::phase_shift_coeff(p, s, z, c); g::adj_phase_shift_coeff(p, s, z, a);
  g::adj_phase_shift_coeff(p, s, z, c);
  g::phase_shift(p, s, 0.1, a, c); g::phase_shift(p, s, 0.1, c); g::adj_phase_shift(p, s, 0.1, a); g::adj_phase_shift(p, s, 0.1, c);
  g::controlled_phase_shift_coeff(p, s, z, a, c); g::controlled_phase_shift_coeff(p, s, z, c);
  g::adj_controlled_phase_shift_coeff(p, s, z, a, c); g::adj_controlled_phase_shift_coeff(p, s, z, c);
  g::controlled_phase_shift(p, s, 0.2, a, c); g::controlled_phase_shift(p, s, 0.2, c);
  g::adj_controlled_phase_shift(p, s, 0.2, a, c); g::adj_controlled_phase_shift(p, s, 0.2, c);
  g::phase_shift2(p, s, 0.1, 0.2, a, c); g::adj_phase_shift2(p, s, 0.1, 0.2, a);
  g::phase_shift3(p, s, 0.1, 0.2, 0.3, a, c); g::adj_phase_shift3(p, s, 0.1, 0.2, 0.3, a);
  g::exponential_pauli_x(p, s, 0.1, a, d); g::adj_exponential_pauli_x(p, s, 0.1, a, c);
  g::exponential_pauli_y(p, s, 0.1, a); g::adj_exponential_pauli_y(p, s, 0.1, a);
  g::exponential_pauli_z(p, s, 0.1, a); g::adj_exponential_pauli_z(p, s, 0.1, a);
  g::swap(p, s, a, d, c); g::adj_swap(p, s, a, d); g::exponential_swap(p, s, 0.1, a, d); g::adj_exponential_swap(p, s, 0.1, a, d, c);
  g::x_rotation_half_pi(p, s, a, c); g::adj_x_rotation_half_pi(p, s, a); g::y_rotation_half_pi(p, s, a); g::adj_y_rotation_half_pi(p, s, a);
  g::sqrt_pauli_x(p, s, a); g::adj_sqrt_pauli_x(p, s, a); g::sqrt_pauli_y(p, s, a); g::adj_sqrt_pauli_y(p, s, a);
  g::sqrt_pauli_z(p, s, a, c); g::adj_sqrt_pauli_z(p, s, a); g::sqrt_pauli_z(p, s, c); g::adj_sqrt_pauli_z(p, s, c);
  g::clear(p, s, a); g::set(p, s, a);
  auto const spins = ket::ranges::all_spin_expectation_values<q_t>(p, s);
  auto const spin = ket::ranges::spin_expectation_value(p, s, a);
  auto const ip = ket::ranges::inner_product(p, s, s);
  auto const f = ket::ranges::fidelity(p, s, s);
  std::mt19937_64 engine{1u};
  std::vector<std::uint64_t> events;
  ket::ranges::generate_events(p, events, s, 4, engine);
  auto const o = g::projective_measurement(p, s, engine, a);
  auto const m = ket::ranges::measure(p, s, engine);
  (void)spins; (void)spin; (void)ip; (void)f; (void)o; (void)m;
}
template void every_gate(rbk::device_state<std::complex<double>>&);
template void every_gate(rbk::device_state<std::complex<float>>&);
"""


@pytest.mark.skipif(not os.path.isdir(KET_INCLUDE) or shutil.which("g++") is None,
                    reason="needs ket's headers and g++ (build machine only)")
def test_adapter_header_compiles_as_cpp14_without_warnings(tmp_path):
    src = tmp_path / "adapter_tu.cpp"
    src.write_text(_HEADER_ONLY_TU)
    cmd = ["g++", "-std=c++14", "-fsyntax-only", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-isystem", KET_INCLUDE, str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


@pytest.mark.skipif(not os.path.isdir(KET_INCLUDE) or shutil.which("g++") is None,
                    reason="needs ket's headers and g++ (build machine only)")
def test_ket_program_selects_device_overloads(tmp_path):
    """The full program compiles against ket's gate headers: a call that fell
    through to ket's CPU templates would fail to compile (device_state has no
    iterators), so success means every call on the device state resolved to
    the overloads of rbk_ket.hpp."""
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-w", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "riken-braket_b200", "bra", "shim"), "-I", KET_INCLUDE,
           os.path.join(ROOT, "tests", "host", "ket_adapter_check.cpp")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


@pytest.mark.gpu
def test_ket_program_on_b200_matches_ket_sequential():
    if not os.path.exists(BINARY):
        pytest.skip("oracle/_ref/ket_adapter_check was not built (ket's headers were absent at build time)")
    r = subprocess.run([BINARY, "20"], capture_output=True, text=True, timeout=600)
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert lines, r.stdout + r.stderr
    for line in lines:
        assert line.get("ok"), line
    assert r.returncode == 0, r.stdout + r.stderr
    cases = {(x["case"], x["qubits"]) for x in lines}
    assert cases == {("complex<double>", 6), ("complex<double>", 14), ("complex<double>", 20),
                     ("complex<float>", 14), ("complex<float>", 20)}
