"""ket::mpi's single-process interface on the device (include/rbk_ket_mpi.hpp).

The same ket::mpi program (tests/host/ket_mpi_check.cpp) runs with ket's own
ket::mpi code -- ket::mpi::state<Complex, false>, the simple_mpi policy and
ket's sequential policy, compiled from ket's headers against the project's
single-process yampi stand-in (oracle/shim/yampi) -- and with the b200 policy
on an rbk::mpi::device_state.  It starts from a non-identity
qubit_permutation and changes it half way (ket::mpi::permutate).  The local
data in ket::mpi's order, the device memory after rbk_state_set_layout, all
spins, the inner product and fidelity must agree to 1e-12 (complex<double>)
/ 2e-5 (complex<float>), and both runs must end with the same permutation.
"""
import json
import os
import shutil
import subprocess

import pytest

from conftest import REFERENCE, ROOT

BINARY = os.path.join(ROOT, "oracle", "_ref", "ket_mpi_check")
KET_INCLUDE = os.path.join(REFERENCE, "ket", "include")
SHIM = os.path.join(ROOT, "oracle", "shim")  # yampi
BSHIM = os.path.join(ROOT, "riken-braket_b200", "bra", "shim")  # Boost
needs_ket = pytest.mark.skipif(not os.path.isdir(KET_INCLUDE) or shutil.which("g++") is None,
                               reason="needs ket's headers and g++ (build machine only)")

_HEADER_TU = r"""
#include <complex>
#include <vector>
#include "rbk_ket_mpi.hpp"
// Instantiates the gate and observable overloads for both precisions.
template <typename Complex>
void every_call(rbk::mpi::device_state<Complex>& s, rbk::mpi::device_state<Complex>& t,
                ket::mpi::qubit_permutation<>& perm, yampi::communicator const& comm, yampi::environment const& env)
{
  namespace g = ket::mpi::gate;
  auto const p = ket::utility::policy::make_b200();
  struct any_mpi_policy { } const mp{};
  std::vector<Complex> buffer;
  ket::qubit<std::uint64_t, unsigned> const a{0u}, b{1u};
  auto const c = ket::make_control(b);
  yampi::datatype const dt{};
  g::hadamard(mp, p, s, perm, buffer, comm, env, a, c);
  g::hadamard(mp, p, s, perm, buffer, dt, comm, env, a);
  g::pauli_x(mp, p, s, perm, buffer, comm, env, a); g::controlled_not(mp, p, s, perm, buffer, comm, env, a, c);
  g::pauli_y(mp, p, s, perm, buffer, comm, env, a); g::pauli_z(mp, p, s, perm, buffer, comm, env, a, c);
  g::phase_shift(mp, p, s, perm, buffer, comm, env, 0.1, a); g::phase_shift2(mp, p, s, perm, buffer, comm, env, 0.1, 0.2, a);
  g::phase_shift3(mp, p, s, perm, buffer, comm, env, 0.1, 0.2, 0.3, a, c);
  g::adj_phase_shift3(mp, p, s, perm, buffer, comm, env, 0.1, 0.2, 0.3, a);
  g::exponential_pauli_y(mp, p, s, perm, buffer, comm, env, 0.1, a);
  g::exponential_pauli_z(mp, p, s, perm, buffer, comm, env, 0.1, a);
  g::swap(mp, p, s, perm, buffer, comm, env, a, b);
  auto const spins = ket::mpi::all_spin_expectation_values<std::allocator<std::array<typename Complex::value_type, 3u>>>(
    mp, p, s, perm, 2u, buffer, comm, env);
  auto const spin = ket::mpi::spin_expectation_value(mp, p, s, perm, buffer, comm, env, a);
  auto const ip = ket::mpi::inner_product(mp, p, s, t, comm, env);
  auto const f = ket::mpi::fidelity(mp, p, s, t, comm, env);
  (void)spins; (void)spin; (void)ip; (void)f;
}
template void every_call(rbk::mpi::device_state<std::complex<double>>&, rbk::mpi::device_state<std::complex<double>>&,
                         ket::mpi::qubit_permutation<>&, yampi::communicator const&, yampi::environment const&);
template void every_call(rbk::mpi::device_state<std::complex<float>>&, rbk::mpi::device_state<std::complex<float>>&,
                         ket::mpi::qubit_permutation<>&, yampi::communicator const&, yampi::environment const&);
"""


@needs_ket
def test_ket_mpi_header_compiles_as_cpp14_without_warnings(tmp_path):
    src = tmp_path / "ket_mpi_tu.cpp"
    src.write_text(_HEADER_TU)
    cmd = ["g++", "-std=c++14", "-fsyntax-only", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-isystem", SHIM, "-isystem", BSHIM, "-isystem", KET_INCLUDE, str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


@needs_ket
def test_ket_mpi_program_compiles_against_the_stand_in(tmp_path):
    """Both runs of the program compile: ket::mpi's own code against the
    single-process yampi stand-in, and the device overloads (a call that fell
    through to ket::mpi's CPU templates would not compile: the device state
    has no iterators)."""
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-w", "-I", os.path.join(ROOT, "include"), "-I", SHIM, "-I", BSHIM,
           "-I", KET_INCLUDE, "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "host", "ket_mpi_check.cpp")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


@needs_ket
def test_yampi_stand_in_runs_ket_mpi_on_the_cpu(tmp_path):
    """ket::mpi's own single-process code runs on the stand-in and gives
    ket's sequential result: H and U3 layers with CNOTs under a permutation,
    compared with the same gates on the data bits the permutation names."""
    src = tmp_path / "stand_in.cpp"
    src.write_text(r"""
#include <complex>
#include <cstdio>
#include <random>
#include <vector>
#include <ket/gate/controlled_not.hpp>
#include <ket/gate/hadamard.hpp>
#include <ket/gate/phase_shift.hpp>
#include <ket/mpi/gate/controlled_not.hpp>
#include <ket/mpi/gate/hadamard.hpp>
#include <ket/mpi/gate/phase_shift.hpp>
#include <ket/mpi/state.hpp>
#include <yampi/environment.hpp>
#include <yampi/communicator.hpp>
int main() {
  using C = std::complex<double>;
  using q_t = ket::qubit<std::uint64_t, unsigned>;
  yampi::environment env{yampi::thread_support::funneled};
  yampi::communicator comm{yampi::tags::world_communicator};
  unsigned const n = 8u;
  std::vector<ket::mpi::permutated<q_t>> map;
  for (unsigned q = 0u; q < n; ++q) map.push_back(ket::mpi::make_permutated(q_t{(q * 3u) % n}));
  ket::mpi::qubit_permutation<> perm(map.begin(), map.end());
  ket::mpi::state<C, false> st{n, std::uint64_t{0}, perm, comm, env};
  std::vector<C> buffer, plain(std::size_t{1} << n);
  plain[0] = 1.0;
  auto const mp = ket::mpi::utility::policy::make_simple_mpi();
  auto const sp = ket::utility::policy::make_sequential();
  std::mt19937_64 rng(3);
  std::uniform_real_distribution<double> u(0.0, 6.0);
  for (unsigned q = 0u; q < n; ++q) {
    ket::mpi::gate::hadamard(mp, sp, st, perm, buffer, comm, env, q_t{q});
    ket::gate::ranges::hadamard(sp, plain, q_t{(q * 3u) % n});
  }
  for (int layer = 0; layer < 4; ++layer) {
    for (unsigned q = 0u; q < n; ++q) {
      double const a = u(rng), b = u(rng), c = u(rng);
      ket::mpi::gate::phase_shift3(mp, sp, st, perm, buffer, comm, env, a, b, c, q_t{q});
      ket::gate::ranges::phase_shift3(sp, plain, a, b, c, q_t{(q * 3u) % n});
    }
    for (unsigned q = layer % 2u; q + 1u < n; q += 2u) {
      ket::mpi::gate::controlled_not(mp, sp, st, perm, buffer, comm, env, q_t{q + 1u}, ket::make_control(q_t{q}));
      ket::gate::ranges::controlled_not(sp, plain, q_t{((q + 1u) * 3u) % n}, ket::make_control(q_t{(q * 3u) % n}));
    }
  }
  double e = 0.0;
  for (std::size_t i = 0; i < plain.size(); ++i) e = std::max(e, std::abs(st[i] - plain[i]));
  std::printf("%.3e\n", e);
  return e == 0.0 ? 0 : 1;
}
""")
    exe = tmp_path / "stand_in"
    cmd = ["g++", "-std=c++17", "-O1", "-w", "-I", SHIM, "-I", BSHIM, "-I", KET_INCLUDE, str(src), "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_ket_mpi_program_on_b200_matches_ket_mpi():
    if not os.path.exists(BINARY):
        pytest.skip("oracle/_ref/ket_mpi_check was not built (ket's headers were absent at build time)")
    r = subprocess.run([BINARY, "20"], capture_output=True, text=True, timeout=600)
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert lines, r.stdout + r.stderr
    for line in lines:
        print(line)
        assert line.get("ok"), line
    assert r.returncode == 0, r.stdout + r.stderr
    cases = {(x["case"], x["qubits"]) for x in lines}
    assert ("complex<double>", 20) in cases and ("complex<float>", 20) in cases
