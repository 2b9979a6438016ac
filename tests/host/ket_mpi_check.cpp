// One program written against ket::mpi's single-process interface, run
// twice: with ket's own ket::mpi code (ket::mpi::state<Complex, false>, the
// simple_mpi policy and ket's sequential policy; compiled from ket's headers
// against the single-process yampi stand-in of oracle/shim) and with the b200
// policy on an rbk::mpi::device_state (include/rbk_ket_mpi.hpp).  The
// gate-calling code is the same function template for both.  The program
// starts from a non-identity qubit_permutation and changes it half way with
// ket::mpi::permutate, as a caller may.  Compared: the local data in
// ket::mpi's order, all spins, the inner product and fidelity of two states,
// and the permutation afterwards.  Prints one JSON line per case and exits 0
// when every case is within tolerance: 1e-12 for complex<double>, 2e-5 for
// complex<float> (both against the complex<double> ket::mpi run).
//
// Build (test infrastructure; needs ket's headers and the stand-ins of
// oracle/shim and riken-braket_b200/bra/shim; links librbk.so and the CUDA runtime, which reads the device
// memory back):  make -C oracle _ref/ket_mpi_check
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <random>
#include <vector>

#include <cuda_runtime.h>

#include <ket/mpi/all_spin_expectation_values.hpp>
#include <ket/mpi/fidelity.hpp>
#include <ket/mpi/gate/controlled_not.hpp>
#include <ket/mpi/gate/controlled_phase_shift.hpp>
#include <ket/mpi/gate/exponential_pauli_x.hpp>
#include <ket/mpi/gate/exponential_pauli_y.hpp>
#include <ket/mpi/gate/exponential_pauli_z.hpp>
#include <ket/mpi/gate/hadamard.hpp>
#include <ket/mpi/gate/not_.hpp>
#include <ket/mpi/gate/pauli_x.hpp>
#include <ket/mpi/gate/pauli_y.hpp>
#include <ket/mpi/gate/pauli_z.hpp>
#include <ket/mpi/gate/phase_shift.hpp>
#include <ket/mpi/gate/swap.hpp>
#include <ket/mpi/gate/toffoli.hpp>
#include <ket/mpi/inner_product.hpp>
#include <ket/mpi/qubit_permutation.hpp>
#include <ket/mpi/state.hpp>
#include <ket/mpi/utility/simple_mpi.hpp>
#include <yampi/communicator.hpp>
#include <yampi/environment.hpp>

#include "rbk_ket_mpi.hpp"

namespace {

using qubit_t = ket::qubit<std::uint64_t, unsigned>;
using permutation_t = ket::mpi::qubit_permutation<std::uint64_t, unsigned>;
using spins_t = std::vector<std::array<double, 3u>>;

// A seeded, non-identity initial permutation.
auto initial_permutation(unsigned const n, std::uint64_t const seed) -> permutation_t
{
  std::vector<ket::mpi::permutated<qubit_t>> map;
  for (unsigned q = 0u; q < n; ++q) map.push_back(ket::mpi::make_permutated(qubit_t{q}));
  std::mt19937_64 rng(seed);
  std::shuffle(map.begin(), map.end(), rng);
  return permutation_t(map.begin(), map.end());
}

// H on every qubit, brick layers of U3 and CNOT, then `mixed` gates cycling
// through the gate families on random distinct qubits; at the middle of the
// mixed gates the program swaps two entries of its permutation.  Angles and
// qubits come from std::mt19937_64(seed), so both runs see the same program.
template <typename Policy, typename State, typename Complex>
void program(Policy const policy, State& state, permutation_t& perm, std::vector<Complex>& buffer,
             yampi::communicator const& comm, yampi::environment const& env, unsigned const n,
             std::uint64_t const seed, int const layers, int const mixed)
{
  namespace g = ket::mpi::gate;
  auto const mp = ket::mpi::utility::policy::make_simple_mpi();
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> angle(0.0, 6.283185307179586);
  auto const q = [](unsigned const b) { return qubit_t{b}; };
  auto const c = [](unsigned const b) { return ket::make_control(qubit_t{b}); };

  for (unsigned i = 0u; i < n; ++i) g::hadamard(mp, policy, state, perm, buffer, comm, env, q(i));
  for (int layer = 0; layer < layers; ++layer) {
    for (unsigned i = 0u; i < n; ++i) {
      double const t = angle(rng), p = angle(rng), l = angle(rng);
      g::phase_shift3(mp, policy, state, perm, buffer, comm, env, t, p, l, q(i));
    }
    for (unsigned i = static_cast<unsigned>(layer) % 2u; i + 1u < n; i += 2u)
      g::controlled_not(mp, policy, state, perm, buffer, comm, env, q(i + 1u), c(i));
  }
  for (int k = 0; k < mixed; ++k) {
    unsigned a = static_cast<unsigned>(rng() % n), b = a, d = a;
    while (b == a) b = static_cast<unsigned>(rng() % n);
    while (d == a || d == b) d = static_cast<unsigned>(rng() % n);
    double const t = angle(rng), p = angle(rng), l = angle(rng);
    std::complex<double> const coeff{std::cos(t), std::sin(t)};
    if (k == mixed / 2) ket::mpi::permutate(perm, q(a), q(b));  // the caller relabels; the local data stays
    switch (k % 14) {
      case 0: g::hadamard(mp, policy, state, perm, buffer, comm, env, q(a), c(b)); break;
      case 1: g::pauli_x(mp, policy, state, perm, buffer, comm, env, q(a)); g::not_(mp, policy, state, perm, buffer, comm, env, q(b), c(d)); break;
      case 2: g::pauli_y(mp, policy, state, perm, buffer, comm, env, q(a)); break;
      case 3: g::pauli_z(mp, policy, state, perm, buffer, comm, env, q(a)); g::pauli_z(mp, policy, state, perm, buffer, comm, env, c(a), c(b)); break;
      case 4: g::phase_shift(mp, policy, state, perm, buffer, comm, env, t, q(a)); break;
      case 5: g::phase_shift_coeff(mp, policy, state, perm, buffer, comm, env, coeff, q(a)); break;
      case 6: g::phase_shift2(mp, policy, state, perm, buffer, comm, env, t, p, q(a)); break;
      case 7: g::phase_shift3(mp, policy, state, perm, buffer, comm, env, t, p, l, q(a), c(b)); break;
      case 8: g::adj_phase_shift3(mp, policy, state, perm, buffer, comm, env, t, p, l, q(d)); break;
      case 9: g::exponential_pauli_x(mp, policy, state, perm, buffer, comm, env, t, q(a)); g::exponential_pauli_y(mp, policy, state, perm, buffer, comm, env, p, q(b)); break;
      case 10: g::exponential_pauli_z(mp, policy, state, perm, buffer, comm, env, t, q(a)); break;
      case 11: g::swap(mp, policy, state, perm, buffer, comm, env, q(a), q(b)); break;
      case 12: g::controlled_phase_shift(mp, policy, state, perm, buffer, comm, env, t, q(a), c(b)); break;
      default: g::not_(mp, policy, state, perm, buffer, comm, env, q(a), c(b), c(d)); g::controlled_not(mp, policy, state, perm, buffer, comm, env, q(d), c(b)); break;
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

auto map_of(permutation_t const& perm, unsigned const n) -> std::vector<unsigned>
{
  std::vector<unsigned> m(n);
  for (unsigned q = 0u; q < n; ++q) m[q] = static_cast<unsigned>(perm[qubit_t{q}].qubit());
  return m;
}

template <typename Complex>
bool run_case(yampi::communicator const& comm, yampi::environment const& env, unsigned const n, int const layers,
              int const mixed, double const tol, char const* name)
{
  auto const cpu = ket::utility::policy::make_sequential();
  auto const gpu = ket::utility::policy::make_b200();
  auto const mp = ket::mpi::utility::policy::make_simple_mpi();
  using ref_state = ket::mpi::state<std::complex<double>, false>;
  using spin_alloc = std::allocator<std::array<double, 3u>>;
  std::uint64_t const init = 5u % (std::uint64_t{1} << n);

  // ket::mpi on the host, complex<double>
  auto perm_cpu = initial_permutation(n, 11u + n);
  std::vector<std::complex<double>> buffer_cpu;
  ref_state want{n, init, perm_cpu, comm, env};
  program(cpu, want, perm_cpu, buffer_cpu, comm, env, n, 7u + n, layers, mixed);
  auto const spins_want = ket::mpi::all_spin_expectation_values<spin_alloc>(mp, cpu, want, perm_cpu, n, buffer_cpu, comm, env);
  auto perm_cpu2 = perm_cpu;
  ref_state want2{n, std::uint64_t{0}, perm_cpu2, comm, env};
  for (unsigned i = 0u; i < n; ++i) ket::mpi::gate::hadamard(mp, cpu, want2, perm_cpu2, buffer_cpu, comm, env, qubit_t{i});
  auto const inner_want = ket::mpi::inner_product(mp, cpu, want, want2, comm, env);
  auto const fid_want = ket::mpi::fidelity(mp, cpu, want, want2, comm, env);

  // the same program on the device
  auto perm_gpu = initial_permutation(n, 11u + n);
  std::vector<Complex> buffer_gpu;
  rbk::mpi::device_state<Complex> got{n, init, perm_gpu, comm, env};
  program(gpu, got, perm_gpu, buffer_gpu, comm, env, n, 7u + n, layers, mixed);
  auto const spins_got = ket::mpi::all_spin_expectation_values<std::allocator<std::array<typename Complex::value_type, 3u>>>(
    mp, gpu, got, perm_gpu, n, buffer_gpu, comm, env);
  auto perm_gpu2 = perm_gpu;
  rbk::mpi::device_state<Complex> got2{n, std::uint64_t{0}, perm_gpu2, comm, env};
  for (unsigned i = 0u; i < n; ++i) ket::mpi::gate::hadamard(mp, gpu, got2, perm_gpu2, buffer_gpu, comm, env, qubit_t{i});
  auto const inner_got = ket::mpi::inner_product(mp, gpu, got, got2, comm, env);
  auto const fid_got = ket::mpi::fidelity(mp, gpu, got, got2, comm, env);

  double const amp_err = max_error(got.local_amplitudes(), want.data());
  double spin_err = 0.0;
  for (unsigned i = 0u; i < n; ++i)
    for (unsigned k = 0u; k < 3u; ++k) spin_err = std::max(spin_err, std::abs(double(spins_got[i][k]) - spins_want[i][k]));
  double const inner_err = std::abs(std::complex<double>(inner_got.real(), inner_got.imag()) - inner_want);
  double const fid_err = std::abs(double(fid_got) - fid_want);
  bool const same_permutation = map_of(perm_cpu, n) == map_of(perm_gpu, n);
  bool identity = true;
  for (unsigned q = 0u; q < n; ++q) identity = identity && map_of(perm_gpu, n)[q] == q;

  // The device memory itself, moved into ket::mpi's order (rbk_state_set_layout)
  // and copied out byte for byte: it must be ket::mpi's local data.
  std::vector<Complex> raw(std::size_t{1} << n);
  void* const device_data = got.device_data();
  double raw_err = 1.0;
  if (cudaMemcpy(raw.data(), device_data, raw.size() * sizeof(Complex), cudaMemcpyDeviceToHost) == cudaSuccess)
    raw_err = max_error(raw, want.data());

  double const worst = std::max({amp_err, spin_err, inner_err, fid_err, raw_err});
  bool const ok = worst <= tol && same_permutation && !identity;
  std::printf("{\"case\": \"%s\", \"qubits\": %u, \"layers\": %d, \"mixed_gates\": %d, \"max_local_data_err\": %.3e, "
              "\"max_spin_err\": %.3e, \"inner_product_err\": %.3e, \"fidelity_err\": %.3e, \"device_memory_err\": %.3e, "
              "\"same_permutation\": %s, \"tol\": %.1e, \"ok\": %s}\n",
              name, n, layers, mixed, amp_err, spin_err, inner_err, fid_err, raw_err, same_permutation ? "true" : "false", tol,
              ok ? "true" : "false");
  std::fflush(stdout);
  return ok;
}

}  // namespace

int main(int argc, char** argv)
{
  yampi::environment env{argc, argv, yampi::thread_support::funneled};
  yampi::communicator comm{yampi::tags::world_communicator};
  unsigned const max_n = argc > 1 ? static_cast<unsigned>(std::atoi(argv[1])) : 20u;
  bool ok = true;
  try {
    for (unsigned const n : {6u, 14u, 20u}) {
      if (n > max_n) continue;
      ok = run_case<std::complex<double>>(comm, env, n, 6, 84, 1e-12, "complex<double>") && ok;
    }
    for (unsigned const n : {14u, 20u}) {
      if (n > max_n) continue;
      ok = run_case<std::complex<float>>(comm, env, n, 6, 84, 2e-5, "complex<float>") && ok;
    }
  } catch (rbk::error const& e) {
    std::printf("{\"error\": \"rbk status %d: %s\", \"ok\": false}\n", e.code(), e.what());
    return 1;
  }
  return ok ? 0 : 1;
}
