// One program written against ket's template API, run twice: with ket's own
// sequential policy on a std::vector (the reference implementation, compiled
// from ket's headers) and with the b200 policy on an rbk::device_state
// (include/rbk_ket.hpp).  The gate-calling code is the same function template
// for both.  Prints one JSON line per case and exits 0 when every case is
// within tolerance: 1e-12 for complex<double>, 2e-5 for complex<float> (both
// against the complex<double> ket run).
//
// Build (test infrastructure; needs ket's headers and the Boost stand-ins of
// riken-braket_b200/bra/shim):  make -C oracle _ref/ket_adapter_check
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <type_traits>
#include <vector>

#include <ket/all_spin_expectation_values.hpp>
#include <ket/fidelity.hpp>
#include <ket/gate/clear.hpp>
#include <ket/gate/projective_measurement.hpp>
#include <ket/gate/controlled_not.hpp>
#include <ket/gate/controlled_phase_shift.hpp>
#include <ket/gate/exponential_pauli_x.hpp>
#include <ket/gate/exponential_pauli_y.hpp>
#include <ket/gate/exponential_pauli_z.hpp>
#include <ket/gate/exponential_swap.hpp>
#include <ket/gate/hadamard.hpp>
#include <ket/gate/not_.hpp>
#include <ket/gate/pauli_x.hpp>
#include <ket/gate/pauli_y.hpp>
#include <ket/gate/pauli_z.hpp>
#include <ket/gate/phase_shift.hpp>
#include <ket/gate/set.hpp>
#include <ket/gate/sqrt_pauli_x.hpp>
#include <ket/gate/sqrt_pauli_y.hpp>
#include <ket/gate/sqrt_pauli_z.hpp>
#include <ket/gate/swap.hpp>
#include <ket/gate/toffoli.hpp>
#include <ket/gate/x_rotation_half_pi.hpp>
#include <ket/gate/y_rotation_half_pi.hpp>
#include <ket/generate_events.hpp>
#include <ket/inner_product.hpp>
#include <ket/measure.hpp>
#include <ket/spin_expectation_value.hpp>
#include <ket/utility/loop_n.hpp>

#include "rbk_ket.hpp"

namespace {

using qubit_t = ket::qubit<std::uint64_t, unsigned>;

// The gate sequence: H on every qubit, brick layers of U3 and CNOT, then
// `mixed` gates cycling through every gate family of rbk_ket.hpp (adjoint
// forms included) on random distinct qubits.  Angles and qubits come from
// std::mt19937_64(seed), so both runs see the same circuit.
template <typename Policy, typename State>
void program(Policy const policy, State& state, unsigned const n, std::uint64_t const seed, int const layers,
             int const mixed)
{
  namespace g = ket::gate::ranges;
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> angle(0.0, 6.283185307179586);
  auto const q = [](unsigned const b) { return qubit_t{b}; };
  auto const c = [](unsigned const b) { return ket::make_control(qubit_t{b}); };

  for (unsigned i = 0u; i < n; ++i) g::hadamard(policy, state, q(i));
  for (int layer = 0; layer < layers; ++layer) {
    for (unsigned i = 0u; i < n; ++i) {
      double const t = angle(rng), p = angle(rng), l = angle(rng);
      g::phase_shift3(policy, state, t, p, l, q(i));
    }
    for (unsigned i = static_cast<unsigned>(layer) % 2u; i + 1u < n; i += 2u) g::controlled_not(policy, state, q(i + 1u), c(i));
  }

  for (int k = 0; k < mixed; ++k) {
    unsigned a = static_cast<unsigned>(rng() % n), b = a, d = a;
    while (b == a) b = static_cast<unsigned>(rng() % n);
    while (d == a || d == b) d = static_cast<unsigned>(rng() % n);
    double const t = angle(rng), p = angle(rng), l = angle(rng);
    std::complex<double> const coeff{std::cos(t), std::sin(t)};
    switch (k % 24) {
      case 0: g::hadamard(policy, state, q(a), c(b)); g::adj_hadamard(policy, state, q(d)); break;
      case 1: g::pauli_x(policy, state, q(a)); g::pauli_x(policy, state, q(a), q(b), c(d)); break;
      case 2: g::pauli_y(policy, state, q(a), c(b)); g::adj_pauli_y(policy, state, q(a), q(b)); break;
      case 3: g::pauli_z(policy, state, q(a), c(b)); g::pauli_z(policy, state, c(a), c(b), c(d)); break;
      case 4: g::pauli_z(policy, state, q(a), q(b)); g::adj_pauli_x(policy, state, q(d), c(a)); break;
      case 5: g::phase_shift_coeff(policy, state, coeff, q(a), c(b)); g::phase_shift_coeff(policy, state, coeff, c(a), c(d)); break;
      case 6: g::phase_shift(policy, state, t, q(a)); g::adj_phase_shift(policy, state, p, q(b), c(d)); break;
      case 7: g::controlled_phase_shift(policy, state, t, q(a), c(b)); g::adj_phase_shift_coeff(policy, state, coeff, q(d)); break;
      case 8: g::controlled_phase_shift_coeff(policy, state, coeff, q(a), c(b)); break;
      case 9: g::phase_shift2(policy, state, t, p, q(a)); g::phase_shift2(policy, state, p, l, q(b), c(d)); break;
      case 10: g::adj_phase_shift2(policy, state, t, p, q(a)); g::adj_phase_shift2(policy, state, p, l, q(b), c(d)); break;
      case 11: g::phase_shift3(policy, state, t, p, l, q(a), c(b)); g::adj_phase_shift3(policy, state, l, t, p, q(d)); break;
      case 12: g::adj_phase_shift3(policy, state, t, p, l, q(a), c(b)); g::phase_shift3(policy, state, p, l, t, q(d)); break;
      case 13: g::exponential_pauli_x(policy, state, t, q(a)); g::exponential_pauli_y(policy, state, p, q(b), c(d)); break;
      case 14: g::exponential_pauli_z(policy, state, t, q(a), q(b)); g::adj_exponential_pauli_x(policy, state, p, q(a), q(d)); break;
      case 15: g::adj_exponential_pauli_y(policy, state, t, q(a)); g::adj_exponential_pauli_z(policy, state, p, q(b), c(d)); break;
      case 16: g::swap(policy, state, q(a), q(b)); g::swap(policy, state, q(a), q(d), c(b)); break;
      case 17: g::exponential_swap(policy, state, t, q(a), q(b)); g::adj_exponential_swap(policy, state, p, q(b), q(d)); break;
      case 18: g::x_rotation_half_pi(policy, state, q(a)); g::adj_y_rotation_half_pi(policy, state, q(b), c(d)); break;
      case 19: g::adj_x_rotation_half_pi(policy, state, q(a), c(b)); g::y_rotation_half_pi(policy, state, q(d)); break;
      case 20: g::sqrt_pauli_x(policy, state, q(a)); g::adj_sqrt_pauli_y(policy, state, q(b), c(d)); break;
      case 21: g::adj_sqrt_pauli_x(policy, state, q(a), c(b)); g::sqrt_pauli_y(policy, state, q(d)); break;
      case 22: g::sqrt_pauli_z(policy, state, q(a), c(b)); g::adj_sqrt_pauli_z(policy, state, c(a), c(d)); break;
      default: g::toffoli(policy, state, q(a), c(b), c(d)); g::not_(policy, state, q(b), c(a)); g::controlled_not(policy, state, q(d), c(b)); break;
    }
  }
}

template <typename Complex>
double max_error(std::vector<Complex> const& got, std::vector<std::complex<double>> const& want)
{
  double e = 0.0;
  for (std::size_t i = 0; i < want.size(); ++i)
    e = std::max(e, std::abs(std::complex<double>(got[i].real(), got[i].imag()) - want[i]));
  return e;
}

// One case: precision Complex on n qubits.  Returns true when within tolerance.
template <typename Complex>
bool run_case(unsigned const n, int const layers, int const mixed, double const tol, char const* name)
{
  auto const policy_cpu = ket::utility::policy::make_sequential();
  auto const policy_gpu = ket::utility::policy::make_b200();
  std::size_t const size = std::size_t{1u} << n;

  // ket on the host, complex<double>
  std::vector<std::complex<double>> want(size), want2(size);
  want[0] = want2[0] = 1.0;
  program(policy_cpu, want, n, 7u + n, layers, mixed);
  program(policy_cpu, want2, n, 1000u + n, layers, mixed / 2);
  auto const spins_want = ket::ranges::all_spin_expectation_values<qubit_t>(policy_cpu, want);
  auto const spin0_want = ket::ranges::spin_expectation_value(policy_cpu, want, qubit_t{n - 1u});
  auto const inner_want = ket::ranges::inner_product(policy_cpu, want, want2);
  auto const fid_want = ket::ranges::fidelity(policy_cpu, want, want2);

  // the same program on the device
  rbk::device_state<Complex> got(n), got2(n);
  program(policy_gpu, got, n, 7u + n, layers, mixed);
  program(policy_gpu, got2, n, 1000u + n, layers, mixed / 2);
  double const amp_err = max_error(got.amplitudes(), want);
  auto const spins_got = ket::ranges::all_spin_expectation_values<qubit_t>(policy_gpu, got);
  double spin_err = 0.0;
  for (unsigned i = 0u; i < n; ++i)
    for (unsigned k = 0u; k < 3u; ++k) spin_err = std::max(spin_err, std::abs(double(spins_got[i][k]) - spins_want[i][k]));
  auto const spin0_got = ket::ranges::spin_expectation_value(policy_gpu, got, qubit_t{n - 1u});
  for (unsigned k = 0u; k < 3u; ++k) spin_err = std::max(spin_err, std::abs(double(spin0_got[k]) - spin0_want[k]));
  auto const inner_got = ket::ranges::inner_product(policy_gpu, got, got2);
  double const inner_err = std::abs(std::complex<double>(inner_got.real(), inner_got.imag()) - inner_want);
  double const fid_err = std::abs(double(ket::ranges::fidelity(policy_gpu, got, got2)) - fid_want);

  // Sampling with the caller's engine (complex<double>: the same events as ket).
  // ket's generate_events overwrites its input with prefix sums, so it gets a copy.
  int sample_mismatches = -1;
  double measured_err = 0.0;
  if (std::is_same<Complex, std::complex<double>>::value) {
    sample_mismatches = 0;
    std::mt19937_64 engine_cpu(99u + n), engine_gpu(99u + n);
    auto copy = want;
    std::vector<std::uint64_t> events_cpu, events_gpu;
    ket::ranges::generate_events(policy_cpu, events_cpu, copy, 64, engine_cpu);
    ket::ranges::generate_events(policy_gpu, events_gpu, got, 64, engine_gpu);
    sample_mismatches += events_cpu.size() == events_gpu.size() ? 0 : 1000;
    for (std::size_t k = 0; k < std::min(events_cpu.size(), events_gpu.size()); ++k)
      sample_mismatches += events_cpu[k] == events_gpu[k] ? 0 : 1;
    auto const outcome_cpu = ket::gate::ranges::projective_measurement(policy_cpu, want, engine_cpu, qubit_t{1u});
    auto const outcome_gpu = ket::gate::ranges::projective_measurement(policy_gpu, got, engine_gpu, qubit_t{1u});
    sample_mismatches += outcome_cpu == outcome_gpu ? 0 : 1;
    measured_err = max_error(got.amplitudes(), want);
    auto measured2 = want2;
    auto const index_cpu = ket::ranges::measure(policy_cpu, measured2, engine_cpu);
    auto const index_gpu = ket::ranges::measure(policy_gpu, got2, engine_gpu);
    sample_mismatches += index_cpu == index_gpu ? 0 : 1;
    measured_err = std::max(measured_err, max_error(got2.amplitudes(), measured2));
  }

  // clear / set, and a state built from host amplitudes
  ket::gate::ranges::clear(policy_cpu, want, qubit_t{0u});
  ket::gate::ranges::set(policy_cpu, want, qubit_t{n - 1u});
  ket::gate::ranges::clear(policy_gpu, got, qubit_t{0u});
  ket::gate::ranges::set(policy_gpu, got, qubit_t{n - 1u});
  double const project_err = max_error(got.amplitudes(), want);
  std::vector<Complex> host(size);
  for (std::size_t i = 0; i < size; ++i) host[i] = Complex(want2[i].real(), want2[i].imag());
  rbk::device_state<Complex> loaded(host);
  double const load_err = max_error(loaded.amplitudes(), want2);

  double const worst = std::max({amp_err, spin_err, inner_err, fid_err, project_err, load_err, measured_err});
  bool const ok = worst <= tol && sample_mismatches <= 0;
  std::printf("{\"case\": \"%s\", \"qubits\": %u, \"layers\": %d, \"mixed_gates\": %d, \"max_amp_err\": %.3e, "
              "\"max_spin_err\": %.3e, \"inner_product_err\": %.3e, \"fidelity_err\": %.3e, \"clear_set_err\": %.3e, "
              "\"upload_err\": %.3e, \"measured_amp_err\": %.3e, \"sample_mismatches\": %d, \"tol\": %.1e, \"ok\": %s}\n",
              name, n, layers, mixed, amp_err, spin_err, inner_err, fid_err, project_err, load_err, measured_err, sample_mismatches, tol,
              ok ? "true" : "false");
  std::fflush(stdout);
  return ok;
}

}  // namespace

int main(int argc, char** argv)
{
  // Optional argument: largest number of qubits (default 20).
  unsigned const max_n = argc > 1 ? static_cast<unsigned>(std::atoi(argv[1])) : 20u;
  bool ok = true;
  try {
    for (unsigned const n : {6u, 14u, 20u}) {
      if (n > max_n) continue;
      ok = run_case<std::complex<double>>(n, 6, 96, 1e-12, "complex<double>") && ok;
    }
    for (unsigned const n : {14u, 20u}) {
      if (n > max_n) continue;
      ok = run_case<std::complex<float>>(n, 6, 96, 2e-5, "complex<float>") && ok;
    }
  } catch (rbk::error const& e) {
    std::printf("{\"error\": \"rbk status %d: %s\", \"ok\": false}\n", e.code(), e.what());
    return 1;
  }
  return ok ? 0 : 1;
}
