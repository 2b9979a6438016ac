/* rbk_ket.hpp -- ket's gate and observable templates on a state held in one
 * B200's HBM.
 *
 * ket, the header-only library under RIKEN-braket, dispatches every gate on a
 * parallel policy and a random-access range of amplitudes, e.g.
 *   ket::gate::ranges::hadamard(policy, state, qubit, controls...)
 * (ket/include/ket/gate/hadamard.hpp:232-249).  This header adds
 *   - one policy, ket::utility::policy::b200 (make_b200()), and
 *   - one range type, rbk::device_state<Complex>, which owns 2^n amplitudes in
 *     device memory through the C ABI of rbk.h,
 * and overloads ket's gate functions (ket::gate::ranges::*, their adj_*
 * forms) and observables (ket::ranges::all_spin_expectation_values,
 * spin_expectation_value, inner_product, fidelity) for that pair.  ket's own policy templates are constrained on
 * ket::utility::policy::meta::is_loop_n_policy, which is false for b200, or
 * are less specialised than the overloads here, so a program written against
 * ket runs on the GPU by passing make_b200() and a device_state where it
 * passed make_sequential()/make_parallel() and a std::vector.
 *
 * Gates are queued and fused as rbk.h describes; every read (amplitudes(),
 * observables) sees all gates issued before it.  Only the qubit and control
 * types of ket are needed (<ket/qubit.hpp>, <ket/control.hpp>); include the
 * ket gate headers as well when the same translation unit also calls ket's
 * CPU implementation.  Errors throw rbk::error (ket itself only asserts;
 * bra's states throw).  Sampling (ket::ranges::generate_events, measure) and
 * ket::gate::ranges::projective_measurement draw from the caller's engine as
 * ket does, one std::uniform_real_distribution<double> value per draw, so an
 * engine shared with ket's CPU code advances identically; unlike ket's
 * generate_events, the state is left intact.
 *
 * C++14 or later.
 */
#ifndef RBK_KET_HPP
#define RBK_KET_HPP

#include <array>
#include <cmath>
#include <cstddef>
#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <random>
#include <type_traits>
#include <utility>
#include <vector>

#include <ket/control.hpp>
#include <ket/qubit.hpp>

#include "rbk.h"

namespace ket {
namespace utility {
namespace policy {
// Execution on one B200 through librbk.so.  The device is chosen when the
// rbk::device_state is created.
struct b200 { };
inline constexpr auto make_b200() noexcept -> b200 { return b200{}; }
}  // namespace policy
}  // namespace utility
}  // namespace ket

namespace ket {
namespace gate {
// ket/include/ket/gate/projective_measurement.hpp:29 defines it; the
// declaration here lets this header name it without that header.
enum class outcome : int;
}  // namespace gate
}  // namespace ket

namespace rbk {

// A failed C ABI call: code() is the rbk_status, what() rbk_last_error().
class error : public std::runtime_error {
 public:
  error(int code, std::string const& message) : std::runtime_error(message), code_(code) { }
  int code() const noexcept { return code_; }

 private:
  int code_;
};

inline void check(int const status)
{
  if (status != RBK_OK) throw error(status, rbk_last_error());
}

namespace detail {
template <typename Complex> struct precision_of;
template <> struct precision_of<std::complex<double>> : std::integral_constant<int, RBK_C128> { };
template <> struct precision_of<std::complex<float>> : std::integral_constant<int, RBK_C64> { };
}  // namespace detail

// 2^n amplitudes of type Complex (std::complex<double> for n <= 33,
// std::complex<float> for n <= 34) in one GPU's HBM: the single-process
// ket::mpi::state<Complex, false> (ket/include/ket/mpi/state.hpp:1973-2100)
// and bra::nompi_state's data_ vector, on the device.  Move-only.
template <typename Complex>
class device_state {
 public:
  using value_type = Complex;
  using real_type = typename Complex::value_type;

  // |initial_index> on `device` (the state ket::mpi::state's constructor and
  // bra's make_initial_data produce).
  explicit device_state(unsigned const num_qubits, std::uint64_t const initial_index = 0u, int const device = 0)
    : num_qubits_{num_qubits}
  {
    check(rbk_state_create(static_cast<int>(num_qubits), detail::precision_of<Complex>::value, initial_index, device,
                           &state_));
  }

  // The amplitudes of a host vector, in logical order; its size must be a power of two.
  explicit device_state(std::vector<Complex> const& amplitudes, int const device = 0)
    : device_state{log2_size(amplitudes.size()), 0u, device}
  {
    assign(amplitudes);
  }

  ~device_state()
  {
    if (state_) rbk_state_destroy(state_);
  }

  device_state(device_state const&) = delete;
  auto operator=(device_state const&) -> device_state& = delete;
  device_state(device_state&& other) noexcept : state_{other.state_}, num_qubits_{other.num_qubits_}
  {
    other.state_ = nullptr;
  }
  auto operator=(device_state&& other) noexcept -> device_state&
  {
    std::swap(state_, other.state_);
    std::swap(num_qubits_, other.num_qubits_);
    return *this;
  }

  auto num_qubits() const noexcept -> unsigned { return num_qubits_; }
  auto size() const noexcept -> std::uint64_t { return std::uint64_t{1u} << num_qubits_; }
  // The C ABI handle, for rbk_* calls this header does not wrap.  A const
  // device_state still executes queued gates when it is read.
  auto handle() const noexcept -> rbk_state* { return state_; }

  // All amplitudes in logical order (qubit q is bit q of the index).
  auto amplitudes() const -> std::vector<Complex>
  {
    std::vector<Complex> result(static_cast<std::size_t>(size()));
    check(rbk_state_download(state_, result.data(), 0u, size()));
    return result;
  }

  auto assign(std::vector<Complex> const& amplitudes) -> void
  {
    if (amplitudes.size() != size()) throw error(RBK_ERR_INVALID, "device_state::assign: size mismatch");
    check(rbk_state_upload(state_, amplitudes.data(), 0u, size()));
  }

  // Drops queued gates and sets the state to |index>.
  auto reset(std::uint64_t const index = 0u) -> void { check(rbk_state_reset(state_, index)); }
  // bra's BEGIN FUSION / END FUSION (bra/src/nompi_state.cpp:1285-1357).
  auto begin_fusion() -> void { check(rbk_begin_fusion(state_)); }
  auto end_fusion() -> void { check(rbk_end_fusion(state_)); }
  // Executes the queued gates and waits for the device.
  auto synchronize() -> void { check(rbk_state_synchronize(state_)); }
  // perm[q]: the physical bit holding logical qubit q (ket::mpi::qubit_permutation).
  auto permutation() const -> std::vector<std::uint32_t>
  {
    std::vector<std::uint32_t> perm(num_qubits_);
    check(rbk_state_get_permutation(state_, perm.data()));
    return perm;
  }

 private:
  static auto log2_size(std::size_t const size) -> unsigned
  {
    unsigned n = 0u;
    while ((std::size_t{1u} << n) < size) ++n;
    if (size == 0u || (std::size_t{1u} << n) != size) throw error(RBK_ERR_INVALID, "device_state: size is not a power of two");
    return n;
  }

  rbk_state* state_ = nullptr;
  unsigned num_qubits_;
};

namespace detail {
// Targets (ket::qubit) and controls (ket::control<ket::qubit>) of a ket
// argument pack, as bit indices.
struct qubit_lists {
  std::vector<std::uint32_t> targets;
  std::vector<std::uint32_t> controls;
};

template <typename StateInteger, typename BitInteger>
inline auto bit(::ket::qubit<StateInteger, BitInteger> const qubit) -> std::uint32_t
{
  return static_cast<std::uint32_t>(static_cast<BitInteger>(qubit));
}

template <typename StateInteger, typename BitInteger>
inline auto collect(qubit_lists& lists, ::ket::qubit<StateInteger, BitInteger> const qubit) -> void
{
  lists.targets.push_back(bit(qubit));
}

template <typename Qubit>
inline auto collect(qubit_lists& lists, ::ket::control<Qubit> const control) -> void
{
  lists.controls.push_back(bit(control.qubit()));
}

template <typename... Qubits>
inline auto split(Qubits const... qubits) -> qubit_lists
{
  qubit_lists lists;
  int const expand[] = {0, (collect(lists, qubits), 0)...};
  static_cast<void>(expand);
  return lists;
}

// Every qubit of the pack, targets first: the set whose all-ones amplitudes a
// diagonal gate (Z, phase shift) multiplies.
template <typename... Qubits>
inline auto all_bits(Qubits const... qubits) -> std::vector<std::uint32_t>
{
  auto lists = split(qubits...);
  lists.targets.insert(lists.targets.end(), lists.controls.begin(), lists.controls.end());
  return lists.targets;
}

inline auto data(std::vector<std::uint32_t> const& v) -> std::uint32_t const* { return v.empty() ? nullptr : v.data(); }
inline auto count(std::vector<std::uint32_t> const& v) -> int { return static_cast<int>(v.size()); }

// exp(i x) as ket::utility::exp_i forms it.
inline auto exp_i(double const x) -> std::complex<double> { return {std::cos(x), std::sin(x)}; }

inline auto apply_matrix(rbk_state* const state, std::complex<double> const m00, std::complex<double> const m01,
                         std::complex<double> const m10, std::complex<double> const m11, std::uint32_t const target,
                         std::vector<std::uint32_t> const& controls) -> void
{
  double const m[8] = {m00.real(), m00.imag(), m01.real(), m01.imag(), m10.real(), m10.imag(), m11.real(), m11.imag()};
  check(rbk_apply_matrix2(state, m, target, data(controls), count(controls)));
}

// One target, or a Pauli string of `letter` on several (with the controls).
inline auto pauli(rbk_state* const state, char const letter, qubit_lists const& lists) -> void
{
  if (lists.targets.size() == 1u) {
    if (letter == 'X') check(rbk_pauli_x(state, lists.targets[0], data(lists.controls), count(lists.controls)));
    else check(rbk_pauli_y(state, lists.targets[0], data(lists.controls), count(lists.controls)));
    return;
  }
  std::string const paulis(lists.targets.size(), letter);
  check(rbk_pauli_string(state, paulis.c_str(), data(lists.targets), count(lists.targets), data(lists.controls),
                         count(lists.controls)));
}

// rbk_uniform_fn over a C++ engine: what ket::utility::positive_random_value_upto
// draws (a uniform_real_distribution on [0, upper)).
template <typename RandomNumberGenerator>
inline double draw_upto(void* const engine, double const upper)
{
  std::uniform_real_distribution<double> distribution{0.0, upper};
  return distribution(*static_cast<RandomNumberGenerator*>(engine));
}

inline auto exponential_pauli(rbk_state* const state, char const letter, double const phase, qubit_lists const& lists)
  -> void
{
  if (lists.targets.size() == 1u) {
    auto const f = letter == 'X' ? rbk_exponential_pauli_x : letter == 'Y' ? rbk_exponential_pauli_y : rbk_exponential_pauli_z;
    check(f(state, phase, lists.targets[0], data(lists.controls), count(lists.controls)));
    return;
  }
  std::string const paulis(lists.targets.size(), letter);
  check(rbk_exponential_pauli_string(state, phase, paulis.c_str(), data(lists.targets), count(lists.targets),
                                     data(lists.controls), count(lists.controls)));
}
}  // namespace detail
}  // namespace rbk

// Gate overloads: each takes (b200, device_state&, the arguments of the ket
// function of the same name) and returns the state, as ket's ranges forms do.
#define RBK_KET_STATE ::rbk::device_state<Complex>
#define RBK_KET_POLICY ::ket::utility::policy::b200 const

namespace ket {
namespace gate {
namespace ranges {

// ---- hadamard.hpp:232-249 ----------------------------------------------------
template <typename Complex, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto hadamard(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,
                     ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  auto const l = ::rbk::detail::split(qubit, control_qubits...);
  ::rbk::check(rbk_hadamard(state.handle(), l.targets[0], ::rbk::detail::data(l.controls), ::rbk::detail::count(l.controls)));
  return state;
}
template <typename Complex, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto adj_hadamard(RBK_KET_POLICY policy, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,
                         ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  return hadamard(policy, state, qubit, control_qubits...);
}

// ---- pauli_x.hpp, not_.hpp:33-51, controlled_not.hpp, toffoli.hpp -------------
// pauli_x(q, qs...): X on every ket::qubit of the pack, controlled by every ket::control.
template <typename Complex, typename StateInteger, typename BitInteger, typename... Qubits>
inline auto pauli_x(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,
                    Qubits const... qubits) -> RBK_KET_STATE&
{
  ::rbk::detail::pauli(state.handle(), 'X', ::rbk::detail::split(qubit, qubits...));
  return state;
}
template <typename Complex, typename StateInteger, typename BitInteger, typename... Qubits>
inline auto adj_pauli_x(RBK_KET_POLICY policy, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,
                        Qubits const... qubits) -> RBK_KET_STATE&
{
  return pauli_x(policy, state, qubit, qubits...);
}
template <typename Complex, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto not_(RBK_KET_POLICY policy, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                 ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  return pauli_x(policy, state, target_qubit, control_qubits...);
}
template <typename Complex, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto adj_not_(RBK_KET_POLICY policy, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                     ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  return pauli_x(policy, state, target_qubit, control_qubits...);
}
template <typename Complex, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto controlled_not(RBK_KET_POLICY policy, RBK_KET_STATE& state,
                           ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                           ::ket::control< ::ket::qubit<StateInteger, BitInteger> > const control_qubit,
                           ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  return pauli_x(policy, state, target_qubit, control_qubit, control_qubits...);
}
template <typename Complex, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto adj_controlled_not(RBK_KET_POLICY policy, RBK_KET_STATE& state,
                               ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                               ::ket::control< ::ket::qubit<StateInteger, BitInteger> > const control_qubit,
                               ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  return pauli_x(policy, state, target_qubit, control_qubit, control_qubits...);
}
template <typename Complex, typename StateInteger, typename BitInteger>
inline auto toffoli(RBK_KET_POLICY policy, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                    ::ket::control< ::ket::qubit<StateInteger, BitInteger> > const control_qubit1,
                    ::ket::control< ::ket::qubit<StateInteger, BitInteger> > const control_qubit2) -> RBK_KET_STATE&
{
  return pauli_x(policy, state, target_qubit, control_qubit1, control_qubit2);
}
template <typename Complex, typename StateInteger, typename BitInteger>
inline auto adj_toffoli(RBK_KET_POLICY policy, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                        ::ket::control< ::ket::qubit<StateInteger, BitInteger> > const control_qubit1,
                        ::ket::control< ::ket::qubit<StateInteger, BitInteger> > const control_qubit2) -> RBK_KET_STATE&
{
  return pauli_x(policy, state, target_qubit, control_qubit1, control_qubit2);
}

// ---- pauli_y.hpp:36-134 -----------------------------------------------------------
template <typename Complex, typename StateInteger, typename BitInteger, typename... Qubits>
inline auto pauli_y(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,
                    Qubits const... qubits) -> RBK_KET_STATE&
{
  ::rbk::detail::pauli(state.handle(), 'Y', ::rbk::detail::split(qubit, qubits...));
  return state;
}
template <typename Complex, typename StateInteger, typename BitInteger, typename... Qubits>
inline auto adj_pauli_y(RBK_KET_POLICY policy, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,
                        Qubits const... qubits) -> RBK_KET_STATE&
{
  return pauli_y(policy, state, qubit, qubits...);
}

// ---- pauli_z.hpp:58-137: Z on each target where every control is one; the
// all-control form negates the amplitudes whose listed qubits are all one. ----
template <typename Complex, typename StateInteger, typename BitInteger, typename... Qubits>
inline auto pauli_z(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,
                    Qubits const... qubits) -> RBK_KET_STATE&
{
  auto const l = ::rbk::detail::split(qubit, qubits...);
  for (auto const target : l.targets) {
    std::vector<std::uint32_t> bits{target};
    bits.insert(bits.end(), l.controls.begin(), l.controls.end());
    ::rbk::check(rbk_pauli_z(state.handle(), bits.data(), ::rbk::detail::count(bits)));
  }
  return state;
}
template <typename Complex, typename... Qubits>
inline auto pauli_z(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::control<Qubits> const... control_qubits) -> RBK_KET_STATE&
{
  auto const bits = ::rbk::detail::all_bits(control_qubits...);
  ::rbk::check(rbk_pauli_z(state.handle(), ::rbk::detail::data(bits), ::rbk::detail::count(bits)));
  return state;
}
template <typename Complex, typename StateInteger, typename BitInteger, typename... Qubits>
inline auto adj_pauli_z(RBK_KET_POLICY policy, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,
                        Qubits const... qubits) -> RBK_KET_STATE&
{
  return pauli_z(policy, state, qubit, qubits...);
}
template <typename Complex, typename... Qubits>
inline auto adj_pauli_z(RBK_KET_POLICY policy, RBK_KET_STATE& state, ::ket::control<Qubits> const... control_qubits)
  -> RBK_KET_STATE&
{
  return pauli_z(policy, state, control_qubits...);
}

// ---- phase_shift.hpp:63-142 (coefficient), :513-521 (phase), and
// controlled_phase_shift.hpp:53-60: the amplitudes whose listed qubits
// (target and controls) are all one are multiplied by the coefficient. ----
template <typename Complex, typename Coefficient, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto phase_shift_coeff(RBK_KET_POLICY, RBK_KET_STATE& state, Coefficient const& phase_coefficient,
                              ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                              ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  auto const bits = ::rbk::detail::all_bits(target_qubit, control_qubits...);
  ::rbk::check(rbk_phase_shift_coeff(state.handle(), static_cast<double>(phase_coefficient.real()),
                                     static_cast<double>(phase_coefficient.imag()), bits.data(), ::rbk::detail::count(bits)));
  return state;
}
template <typename Complex, typename Coefficient, typename... Qubits>
inline auto phase_shift_coeff(RBK_KET_POLICY, RBK_KET_STATE& state, Coefficient const& phase_coefficient,
                              ::ket::control<Qubits> const... control_qubits) -> RBK_KET_STATE&
{
  auto const bits = ::rbk::detail::all_bits(control_qubits...);
  ::rbk::check(rbk_phase_shift_coeff(state.handle(), static_cast<double>(phase_coefficient.real()),
                                     static_cast<double>(phase_coefficient.imag()), ::rbk::detail::data(bits),
                                     ::rbk::detail::count(bits)));
  return state;
}
template <typename Complex, typename Coefficient, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto adj_phase_shift_coeff(RBK_KET_POLICY policy, RBK_KET_STATE& state, Coefficient const& phase_coefficient,
                                  ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                                  ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  return phase_shift_coeff(policy, state, std::conj(phase_coefficient), target_qubit, control_qubits...);
}
template <typename Complex, typename Coefficient, typename... Qubits>
inline auto adj_phase_shift_coeff(RBK_KET_POLICY policy, RBK_KET_STATE& state, Coefficient const& phase_coefficient,
                                  ::ket::control<Qubits> const... control_qubits) -> RBK_KET_STATE&
{
  return phase_shift_coeff(policy, state, std::conj(phase_coefficient), control_qubits...);
}

template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto phase_shift(RBK_KET_POLICY, RBK_KET_STATE& state, Real const phase,
                        ::ket::qubit<StateInteger, BitInteger> const target_qubit, ControlQubits const... control_qubits)
  -> std::enable_if_t<std::is_arithmetic<Real>::value, RBK_KET_STATE&>
{
  auto const bits = ::rbk::detail::all_bits(target_qubit, control_qubits...);
  ::rbk::check(rbk_phase_shift(state.handle(), static_cast<double>(phase), bits.data(), ::rbk::detail::count(bits)));
  return state;
}
template <typename Complex, typename Real, typename... Qubits>
inline auto phase_shift(RBK_KET_POLICY, RBK_KET_STATE& state, Real const phase, ::ket::control<Qubits> const... control_qubits)
  -> std::enable_if_t<std::is_arithmetic<Real>::value, RBK_KET_STATE&>
{
  auto const bits = ::rbk::detail::all_bits(control_qubits...);
  ::rbk::check(rbk_phase_shift(state.handle(), static_cast<double>(phase), ::rbk::detail::data(bits), ::rbk::detail::count(bits)));
  return state;
}
template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto adj_phase_shift(RBK_KET_POLICY policy, RBK_KET_STATE& state, Real const phase,
                            ::ket::qubit<StateInteger, BitInteger> const target_qubit, ControlQubits const... control_qubits)
  -> std::enable_if_t<std::is_arithmetic<Real>::value, RBK_KET_STATE&>
{
  return phase_shift(policy, state, -phase, target_qubit, control_qubits...);
}
template <typename Complex, typename Real, typename... Qubits>
inline auto adj_phase_shift(RBK_KET_POLICY policy, RBK_KET_STATE& state, Real const phase,
                            ::ket::control<Qubits> const... control_qubits)
  -> std::enable_if_t<std::is_arithmetic<Real>::value, RBK_KET_STATE&>
{
  return phase_shift(policy, state, -phase, control_qubits...);
}

template <typename Complex, typename Coefficient, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto controlled_phase_shift_coeff(RBK_KET_POLICY policy, RBK_KET_STATE& state, Coefficient const& phase_coefficient,
                                         ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                                         ::ket::control< ::ket::qubit<StateInteger, BitInteger> > const control_qubit,
                                         ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  return phase_shift_coeff(policy, state, phase_coefficient, target_qubit, control_qubit, control_qubits...);
}
template <typename Complex, typename Coefficient, typename... Qubits>
inline auto controlled_phase_shift_coeff(RBK_KET_POLICY policy, RBK_KET_STATE& state, Coefficient const& phase_coefficient,
                                         ::ket::control<Qubits> const... control_qubits) -> RBK_KET_STATE&
{
  return phase_shift_coeff(policy, state, phase_coefficient, control_qubits...);
}
template <typename Complex, typename Coefficient, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto adj_controlled_phase_shift_coeff(RBK_KET_POLICY policy, RBK_KET_STATE& state,
                                             Coefficient const& phase_coefficient,
                                             ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                                             ::ket::control< ::ket::qubit<StateInteger, BitInteger> > const control_qubit,
                                             ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  return phase_shift_coeff(policy, state, std::conj(phase_coefficient), target_qubit, control_qubit, control_qubits...);
}
template <typename Complex, typename Coefficient, typename... Qubits>
inline auto adj_controlled_phase_shift_coeff(RBK_KET_POLICY policy, RBK_KET_STATE& state,
                                             Coefficient const& phase_coefficient,
                                             ::ket::control<Qubits> const... control_qubits) -> RBK_KET_STATE&
{
  return phase_shift_coeff(policy, state, std::conj(phase_coefficient), control_qubits...);
}
template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto controlled_phase_shift(RBK_KET_POLICY policy, RBK_KET_STATE& state, Real const phase,
                                   ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                                   ::ket::control< ::ket::qubit<StateInteger, BitInteger> > const control_qubit,
                                   ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  return phase_shift(policy, state, phase, target_qubit, control_qubit, control_qubits...);
}
template <typename Complex, typename Real, typename... Qubits>
inline auto controlled_phase_shift(RBK_KET_POLICY policy, RBK_KET_STATE& state, Real const phase,
                                   ::ket::control<Qubits> const... control_qubits) -> RBK_KET_STATE&
{
  return phase_shift(policy, state, phase, control_qubits...);
}
template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto adj_controlled_phase_shift(RBK_KET_POLICY policy, RBK_KET_STATE& state, Real const phase,
                                       ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                                       ::ket::control< ::ket::qubit<StateInteger, BitInteger> > const control_qubit,
                                       ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  return phase_shift(policy, state, -phase, target_qubit, control_qubit, control_qubits...);
}
template <typename Complex, typename Real, typename... Qubits>
inline auto adj_controlled_phase_shift(RBK_KET_POLICY policy, RBK_KET_STATE& state, Real const phase,
                                       ::ket::control<Qubits> const... control_qubits) -> RBK_KET_STATE&
{
  return phase_shift(policy, state, -phase, control_qubits...);
}

// ---- U2 and U3: phase_shift2 (phase_shift.hpp:660-709), phase_shift3
// (:1200-1332).  The adjoints are the matrices of ket's adj_phase_shift2
// (:931-979) and adj_phase_shift3 (:1494-1552), built in double precision. ----
template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto phase_shift2(RBK_KET_POLICY, RBK_KET_STATE& state, Real const phase1, Real const phase2,
                         ::ket::qubit<StateInteger, BitInteger> const target_qubit, ControlQubits const... control_qubits)
  -> RBK_KET_STATE&
{
  auto const l = ::rbk::detail::split(target_qubit, control_qubits...);
  ::rbk::check(rbk_phase_shift2(state.handle(), static_cast<double>(phase1), static_cast<double>(phase2), l.targets[0],
                                ::rbk::detail::data(l.controls), ::rbk::detail::count(l.controls)));
  return state;
}
template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto adj_phase_shift2(RBK_KET_POLICY, RBK_KET_STATE& state, Real const phase1, Real const phase2,
                             ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                             ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  auto const l = ::rbk::detail::split(target_qubit, control_qubits...);
  double const r = 0.70710678118654752440084436210484903928483593768847;  // 1/sqrt(2), correctly rounded
  auto const c1 = ::rbk::detail::exp_i(-static_cast<double>(phase1));
  auto const c2 = ::rbk::detail::exp_i(-static_cast<double>(phase2));
  ::rbk::detail::apply_matrix(state.handle(), {r, 0.0}, r * c1, -r * c2, r * c1 * c2, l.targets[0], l.controls);
  return state;
}
template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto phase_shift3(RBK_KET_POLICY, RBK_KET_STATE& state, Real const phase1, Real const phase2, Real const phase3,
                         ::ket::qubit<StateInteger, BitInteger> const target_qubit, ControlQubits const... control_qubits)
  -> RBK_KET_STATE&
{
  auto const l = ::rbk::detail::split(target_qubit, control_qubits...);
  ::rbk::check(rbk_phase_shift3(state.handle(), static_cast<double>(phase1), static_cast<double>(phase2),
                                static_cast<double>(phase3), l.targets[0], ::rbk::detail::data(l.controls),
                                ::rbk::detail::count(l.controls)));
  return state;
}
template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto adj_phase_shift3(RBK_KET_POLICY, RBK_KET_STATE& state, Real const phase1, Real const phase2, Real const phase3,
                             ::ket::qubit<StateInteger, BitInteger> const target_qubit,
                             ControlQubits const... control_qubits) -> RBK_KET_STATE&
{
  auto const l = ::rbk::detail::split(target_qubit, control_qubits...);
  double const sine = std::sin(0.5 * static_cast<double>(phase1));
  double const cosine = std::cos(0.5 * static_cast<double>(phase1));
  auto const c2 = ::rbk::detail::exp_i(-static_cast<double>(phase2));
  auto const c3 = ::rbk::detail::exp_i(-static_cast<double>(phase3));
  ::rbk::detail::apply_matrix(state.handle(), {cosine, 0.0}, sine * c2, -sine * c3, cosine * c2 * c3, l.targets[0],
                              l.controls);
  return state;
}

// ---- exponential_pauli_{x,y,z}.hpp: exp(i theta P) on one target, or on the
// Pauli product over several targets, with controls. ----
#define RBK_KET_EXPONENTIAL_PAULI(NAME, LETTER)                                                                       \
  template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... Qubits>         \
  inline auto NAME(RBK_KET_POLICY, RBK_KET_STATE& state, Real const phase,                                          \
                   ::ket::qubit<StateInteger, BitInteger> const qubit, Qubits const... qubits)                       \
    -> std::enable_if_t<std::is_arithmetic<Real>::value, RBK_KET_STATE&>                                          \
  {                                                                                                                  \
    ::rbk::detail::exponential_pauli(state.handle(), LETTER, static_cast<double>(phase),                            \
                                     ::rbk::detail::split(qubit, qubits...));                                       \
    return state;                                                                                                    \
  }                                                                                                                  \
  template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... Qubits>         \
  inline auto adj_##NAME(RBK_KET_POLICY, RBK_KET_STATE& state, Real const phase,                                    \
                         ::ket::qubit<StateInteger, BitInteger> const qubit, Qubits const... qubits)                 \
    -> std::enable_if_t<std::is_arithmetic<Real>::value, RBK_KET_STATE&>                                          \
  {                                                                                                                  \
    ::rbk::detail::exponential_pauli(state.handle(), LETTER, -static_cast<double>(phase),                           \
                                     ::rbk::detail::split(qubit, qubits...));                                       \
    return state;                                                                                                    \
  }
RBK_KET_EXPONENTIAL_PAULI(exponential_pauli_x, 'X')
RBK_KET_EXPONENTIAL_PAULI(exponential_pauli_y, 'Y')
RBK_KET_EXPONENTIAL_PAULI(exponential_pauli_z, 'Z')
#undef RBK_KET_EXPONENTIAL_PAULI

// ---- swap.hpp:34-75 (uncontrolled swaps only relabel the layout map) and
// exponential_swap.hpp:37-40, :103 ----
template <typename Complex, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto swap(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const target_qubit1,
                 ::ket::qubit<StateInteger, BitInteger> const target_qubit2, ControlQubits const... control_qubits)
  -> RBK_KET_STATE&
{
  auto const l = ::rbk::detail::split(target_qubit1, target_qubit2, control_qubits...);
  ::rbk::check(rbk_swap(state.handle(), l.targets[0], l.targets[1], ::rbk::detail::data(l.controls),
                        ::rbk::detail::count(l.controls)));
  return state;
}
template <typename Complex, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto adj_swap(RBK_KET_POLICY policy, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const target_qubit1,
                     ::ket::qubit<StateInteger, BitInteger> const target_qubit2, ControlQubits const... control_qubits)
  -> RBK_KET_STATE&
{
  return swap(policy, state, target_qubit1, target_qubit2, control_qubits...);
}
template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto exponential_swap(RBK_KET_POLICY, RBK_KET_STATE& state, Real const phase,
                             ::ket::qubit<StateInteger, BitInteger> const target_qubit1,
                             ::ket::qubit<StateInteger, BitInteger> const target_qubit2,
                             ControlQubits const... control_qubits)
  -> std::enable_if_t<std::is_arithmetic<Real>::value, RBK_KET_STATE&>
{
  auto const l = ::rbk::detail::split(target_qubit1, target_qubit2, control_qubits...);
  ::rbk::check(rbk_exponential_swap(state.handle(), static_cast<double>(phase), l.targets[0], l.targets[1],
                                    ::rbk::detail::data(l.controls), ::rbk::detail::count(l.controls)));
  return state;
}
template <typename Complex, typename Real, typename StateInteger, typename BitInteger, typename... ControlQubits>
inline auto adj_exponential_swap(RBK_KET_POLICY policy, RBK_KET_STATE& state, Real const phase,
                                 ::ket::qubit<StateInteger, BitInteger> const target_qubit1,
                                 ::ket::qubit<StateInteger, BitInteger> const target_qubit2,
                                 ControlQubits const... control_qubits)
  -> std::enable_if_t<std::is_arithmetic<Real>::value, RBK_KET_STATE&>
{
  return exponential_swap(policy, state, -phase, target_qubit1, target_qubit2, control_qubits...);
}

// ---- x_rotation_half_pi.hpp:34, :254; y_rotation_half_pi.hpp:33, :251;
// sqrt_pauli_x.hpp:32, :259; sqrt_pauli_y.hpp:33, :256 ----
#define RBK_KET_HALF_PI_GATE(NAME, CALL)                                                                              \
  template <typename Complex, typename StateInteger, typename BitInteger, typename... ControlQubits>                 \
  inline auto NAME(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,        \
                   ControlQubits const... control_qubits) -> RBK_KET_STATE&                                         \
  {                                                                                                                  \
    auto const l = ::rbk::detail::split(qubit, control_qubits...);                                                  \
    ::rbk::check(CALL(state.handle(), 0, l.targets[0], ::rbk::detail::data(l.controls),                            \
                      ::rbk::detail::count(l.controls)));                                                            \
    return state;                                                                                                    \
  }                                                                                                                  \
  template <typename Complex, typename StateInteger, typename BitInteger, typename... ControlQubits>                 \
  inline auto adj_##NAME(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,  \
                         ControlQubits const... control_qubits) -> RBK_KET_STATE&                                   \
  {                                                                                                                  \
    auto const l = ::rbk::detail::split(qubit, control_qubits...);                                                  \
    ::rbk::check(CALL(state.handle(), 1, l.targets[0], ::rbk::detail::data(l.controls),                            \
                      ::rbk::detail::count(l.controls)));                                                            \
    return state;                                                                                                    \
  }
RBK_KET_HALF_PI_GATE(x_rotation_half_pi, rbk_x_rotation_half_pi)
RBK_KET_HALF_PI_GATE(y_rotation_half_pi, rbk_y_rotation_half_pi)
RBK_KET_HALF_PI_GATE(sqrt_pauli_x, rbk_sqrt_pauli_x)
RBK_KET_HALF_PI_GATE(sqrt_pauli_y, rbk_sqrt_pauli_y)
#undef RBK_KET_HALF_PI_GATE

// ---- sqrt_pauli_z.hpp:55-205, :428-520: i (adjoint: -i) on |1> of each
// target where every control is one; the all-control form on |1...1>. ----
template <typename Complex, typename StateInteger, typename BitInteger, typename... Qubits>
inline auto sqrt_pauli_z(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,
                         Qubits const... qubits) -> RBK_KET_STATE&
{
  auto const l = ::rbk::detail::split(qubit, qubits...);
  ::rbk::check(rbk_sqrt_pauli_z(state.handle(), 0, l.targets.data(), ::rbk::detail::count(l.targets),
                                ::rbk::detail::data(l.controls), ::rbk::detail::count(l.controls)));
  return state;
}
template <typename Complex, typename StateInteger, typename BitInteger, typename... Qubits>
inline auto adj_sqrt_pauli_z(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit,
                             Qubits const... qubits) -> RBK_KET_STATE&
{
  auto const l = ::rbk::detail::split(qubit, qubits...);
  ::rbk::check(rbk_sqrt_pauli_z(state.handle(), 1, l.targets.data(), ::rbk::detail::count(l.targets),
                                ::rbk::detail::data(l.controls), ::rbk::detail::count(l.controls)));
  return state;
}
template <typename Complex, typename Qubit, typename... Qubits>
inline auto sqrt_pauli_z(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::control<Qubit> const control_qubit,
                         ::ket::control<Qubits> const... control_qubits) -> RBK_KET_STATE&
{
  auto const bits = ::rbk::detail::all_bits(control_qubit, control_qubits...);
  ::rbk::check(rbk_sqrt_pauli_z(state.handle(), 0, bits.data(), 1, bits.data() + 1, ::rbk::detail::count(bits) - 1));
  return state;
}
template <typename Complex, typename Qubit, typename... Qubits>
inline auto adj_sqrt_pauli_z(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::control<Qubit> const control_qubit,
                             ::ket::control<Qubits> const... control_qubits) -> RBK_KET_STATE&
{
  auto const bits = ::rbk::detail::all_bits(control_qubit, control_qubits...);
  ::rbk::check(rbk_sqrt_pauli_z(state.handle(), 1, bits.data(), 1, bits.data() + 1, ::rbk::detail::count(bits) - 1));
  return state;
}

// ---- clear.hpp / set.hpp: project the qubit onto |0> / |1> and renormalise ----
template <typename Complex, typename StateInteger, typename BitInteger>
inline auto clear(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit) -> RBK_KET_STATE&
{
  ::rbk::check(rbk_clear(state.handle(), ::rbk::detail::bit(qubit)));
  return state;
}
template <typename Complex, typename StateInteger, typename BitInteger>
inline auto set(RBK_KET_POLICY, RBK_KET_STATE& state, ::ket::qubit<StateInteger, BitInteger> const qubit) -> RBK_KET_STATE&
{
  ::rbk::check(rbk_set(state.handle(), ::rbk::detail::bit(qubit)));
  return state;
}

// ---- projective_measurement.hpp:154-186: outcome 0 when a draw on [0, p0 + p1)
// from the caller's engine falls below p0; the kept half is scaled by p^(-1/2). ----
template <typename Complex, typename RandomNumberGenerator, typename StateInteger, typename BitInteger>
inline auto projective_measurement(RBK_KET_POLICY, RBK_KET_STATE& state, RandomNumberGenerator& random_number_generator,
                                   ::ket::qubit<StateInteger, BitInteger> const qubit) -> ::ket::gate::outcome
{
  int one = 0;
  ::rbk::check(rbk_projective_measurement_with(state.handle(), ::rbk::detail::bit(qubit),
                                               &::rbk::detail::draw_upto<RandomNumberGenerator>,
                                               static_cast<void*>(&random_number_generator), &one));
  return static_cast< ::ket::gate::outcome>(one);
}

}  // namespace ranges
}  // namespace gate

// ---- observables (ket::ranges, the range forms of ket's observables) ---------------
namespace ranges {

// <S_x>, <S_y>, <S_z> of every qubit in spin-1/2 units, qubit order
// (ket/include/ket/all_spin_expectation_values.hpp:22-42): one tiled read of
// the state serves many qubits.
template <typename Qubit, typename Complex>
inline auto all_spin_expectation_values(RBK_KET_POLICY, RBK_KET_STATE const& state)
  -> std::vector<std::array<typename Complex::value_type, 3u>>
{
  std::vector<double> spins(3u * state.num_qubits());
  ::rbk::check(rbk_spin_expectation_values(state.handle(), spins.data()));
  std::vector<std::array<typename Complex::value_type, 3u>> result(state.num_qubits());
  for (unsigned q = 0u; q < state.num_qubits(); ++q)
    for (unsigned k = 0u; k < 3u; ++k) result[q][k] = static_cast<typename Complex::value_type>(spins[3u * q + k]);
  return result;
}

// spin_expectation_value.hpp:21-80 for one qubit: half the Pauli X, Y, Z expectation values.
template <typename Complex, typename StateInteger, typename BitInteger>
inline auto spin_expectation_value(RBK_KET_POLICY, RBK_KET_STATE const& state,
                                   ::ket::qubit<StateInteger, BitInteger> const qubit)
  -> std::array<typename Complex::value_type, 3u>
{
  unsigned const n = state.num_qubits();
  auto const q = ::rbk::detail::bit(qubit);
  std::string strings(3u * n, 'I');
  strings[q] = 'X';
  strings[n + q] = 'Y';
  strings[2u * n + q] = 'Z';
  std::array<typename Complex::value_type, 3u> result{};
  for (unsigned k = 0u; k < 3u; ++k) {
    double const coeff[2] = {0.5, 0.0};
    double value[2] = {0.0, 0.0};
    ::rbk::check(rbk_expectation_pauli(state.handle(), 1, strings.c_str() + k * n, coeff, value));
    result[k] = static_cast<typename Complex::value_type>(value[0]);
  }
  return result;
}

// inner_product.hpp:30-56: <state2|state1> = sum conj(state2_i) state1_i.
template <typename Complex>
inline auto inner_product(RBK_KET_POLICY, RBK_KET_STATE const& state1, RBK_KET_STATE const& state2) -> Complex
{
  double value[2] = {0.0, 0.0};
  ::rbk::check(rbk_inner_product(state1.handle(), state2.handle(), value));
  return Complex(static_cast<typename Complex::value_type>(value[0]), static_cast<typename Complex::value_type>(value[1]));
}

// fidelity.hpp: |<state2|state1>|^2.
template <typename Complex>
inline auto fidelity(RBK_KET_POLICY, RBK_KET_STATE const& state1, RBK_KET_STATE const& state2) -> typename Complex::value_type
{
  double value = 0.0;
  ::rbk::check(rbk_fidelity(state1.handle(), state2.handle(), &value));
  return static_cast<typename Complex::value_type>(value);
}

// generate_events.hpp:18-48, 102-113: num_events basis-state indices drawn
// from |a_i|^2 with the caller's engine, into result (cleared first).
template <typename Complex, typename StateInteger, typename Allocator, typename RandomNumberGenerator>
inline auto generate_events(RBK_KET_POLICY, std::vector<StateInteger, Allocator>& result, RBK_KET_STATE& state,
                            int const num_events, RandomNumberGenerator& random_number_generator) -> void
{
  std::vector<std::uint64_t> events(static_cast<std::size_t>(num_events > 0 ? num_events : 0));
  ::rbk::check(rbk_generate_events_with(state.handle(), num_events, &::rbk::detail::draw_upto<RandomNumberGenerator>,
                                        static_cast<void*>(&random_number_generator), events.data()));
  result.assign(events.begin(), events.end());
}

// measure.hpp:16-46, 56-66: one index drawn from |a_i|^2 with the caller's
// engine; the state becomes that basis state.
template <typename Complex, typename RandomNumberGenerator>
inline auto measure(RBK_KET_POLICY, RBK_KET_STATE& state, RandomNumberGenerator& random_number_generator) -> std::ptrdiff_t
{
  std::uint64_t index = 0u;
  ::rbk::check(rbk_measure_with(state.handle(), &::rbk::detail::draw_upto<RandomNumberGenerator>,
                                static_cast<void*>(&random_number_generator), &index));
  return static_cast<std::ptrdiff_t>(index);
}

}  // namespace ranges
}  // namespace ket

#undef RBK_KET_POLICY
#undef RBK_KET_STATE

#endif  // RBK_KET_HPP
