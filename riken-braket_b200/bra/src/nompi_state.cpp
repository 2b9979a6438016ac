// The B200 bra::nompi_state (include/bra/nompi_state.hpp in this directory):
// bra::state's do_* backend (bra/include/bra/state.hpp:1022-1318) on an rbk
// engine state.  Each gate becomes one C ABI call (include/rbk.h); the engine
// queues it and runs the queue as fused passes when a result is read.  The
// multi-circuit instructions keep bra's protocol: a do_* call that needs
// another circuit marks the state as waiting with a wait_reason, and bra's
// main then calls the free functions at the end of this file for the waiting
// states.
#include <bra/nompi_state.hpp>

#include <cctype>
#include <complex>
#include <cstdlib>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <boost/algorithm/string/case_conv.hpp>
#include <boost/lexical_cast.hpp>

namespace bra {
namespace {

void check(int const rc)
{
  if (rc != RBK_OK) throw std::runtime_error(std::string{"B200 engine: "} + rbk_last_error());
}

std::uint32_t bit(::bra::qubit_type const qubit)
{
  return static_cast<std::uint32_t>(static_cast< ::bra::bit_integer_type>(qubit));
}
std::uint32_t bit(::bra::control_qubit_type const control) { return bit(control.qubit()); }

std::vector<std::uint32_t> bits(std::vector< ::bra::qubit_type > const& qubits)
{
  std::vector<std::uint32_t> result;
  for (auto const q : qubits) result.push_back(bit(q));
  return result;
}
std::vector<std::uint32_t> bits(std::vector< ::bra::control_qubit_type > const& controls)
{
  std::vector<std::uint32_t> result;
  for (auto const c : controls) result.push_back(bit(c));
  return result;
}
std::vector<std::uint32_t> bits(std::initializer_list< ::bra::control_qubit_type > const controls)
{
  return bits(std::vector< ::bra::control_qubit_type >(controls));
}

int size_of(std::vector<std::uint32_t> const& v) { return static_cast<int>(v.size()); }

// What ket::utility::positive_random_value_upto draws from the engine (a
// uniform_real_distribution on [0, upper)), as the engine's sampling calls it.
double draw_upto(void* const engine, double const upper)
{
  std::uniform_real_distribution<double> distribution{0.0, upper};
  return distribution(*static_cast<std::mt19937_64*>(engine));
}

constexpr double kHalfPi = 1.570796326794896619231321691639751442;

// The engine's Pauli-sum format: one string of all n qubits per term, the
// term's k-th letter on the k-th operated qubit; coefficients as (re, im).
void operator_terms(::bra::pauli_string_space const& op, std::vector< ::bra::qubit_type > const& operated_qubits,
                    unsigned const num_qubits, std::string& strings, std::vector<double>& coeffs)
{
  for (auto const& term : op) {
    std::string full(num_qubits, 'I');
    for (std::size_t k = 0; k < operated_qubits.size(); ++k) full[bit(operated_qubits[k])] = term.first[k];
    strings += full;
    coeffs.push_back(term.second.real());
    coeffs.push_back(term.second.imag());
  }
}

}  // namespace

nompi_state::nompi_state(::bra::state::state_integer_type const initial_integer, unsigned int const total_num_qubits,
                         unsigned int const /*num_threads*/, ::bra::state::seed_type const seed,
                         bool const is_depolarizing_channel, ::bra::real_type const depolarizing_px,
                         ::bra::real_type const depolarizing_py, ::bra::real_type const depolarizing_pz,
                         bool const uses_depolarizing_seed, ::bra::state::seed_type const depolarizing_seed,
                         int const circuit_index)
  : ::bra::state{total_num_qubits, seed, is_depolarizing_channel, depolarizing_px, depolarizing_py, depolarizing_pz,
                 uses_depolarizing_seed, depolarizing_seed, circuit_index}
{
  char const* const device = std::getenv("RBK_DEVICE");
  check(rbk_state_create(static_cast<int>(total_num_qubits), RBK_C128, initial_integer, device ? std::atoi(device) : 0,
                         &handle_));
}

nompi_state::~nompi_state()
{
  if (handle_) rbk_state_destroy(handle_);
}

nompi_state::nompi_state(nompi_state&& other) noexcept
  : ::bra::state{std::move(other)}, handle_{other.handle_}, is_waiting_{other.is_waiting_}
{
  other.handle_ = nullptr;
}

nompi_state& nompi_state::operator=(nompi_state&& other) noexcept
{
  ::bra::state::operator=(std::move(other));
  std::swap(handle_, other.handle_);
  is_waiting_ = other.is_waiting_;
  return *this;
}

// ---- the multi-circuit protocol ------------------------------------------------

auto nompi_state::do_is_waiting() const -> bool { return is_waiting_; }
auto nompi_state::do_cancel_waiting() -> void { is_waiting_ = false; }

// A uniform value on [0, 1) for the depolarizing channel, from its own
// generator when it was given a seed.
auto nompi_state::generate_probability() -> real_type
{
  std::uniform_real_distribution<double> distribution{0.0, 1.0};
  return static_cast<real_type>(uses_depolarizing_seed_ ? distribution(depolarizing_random_number_generator_)
                                                        : distribution(random_number_generator_));
}

#define RBK_WAIT_PEER(NAME, TAG)                                                                                        \
  auto nompi_state::NAME(int const other_circuit_index, std::string const& variable_name, int const num_elements)     \
    RBK_CONST_##NAME->void                                                                                            \
  {                                                                                                                   \
    if (other_circuit_index < 0 || other_circuit_index == circuit_index_) return;                                     \
    is_waiting_ = true;                                                                                               \
    wait_reason_ = ::bra::wait_reason{::bra::wait_reason::TAG{}, other_circuit_index, variable_name, num_elements};   \
  }
#define RBK_CONST_do_send_real_variable const
#define RBK_CONST_do_send_complex_variable const
#define RBK_CONST_do_send_int_variable const
#define RBK_CONST_do_receive_real_variable
#define RBK_CONST_do_receive_complex_variable
#define RBK_CONST_do_receive_int_variable
RBK_WAIT_PEER(do_send_real_variable, send_real_variable_t)
RBK_WAIT_PEER(do_send_complex_variable, send_complex_variable_t)
RBK_WAIT_PEER(do_send_int_variable, send_int_variable_t)
RBK_WAIT_PEER(do_receive_real_variable, receive_real_variable_t)
RBK_WAIT_PEER(do_receive_complex_variable, receive_complex_variable_t)
RBK_WAIT_PEER(do_receive_int_variable, receive_int_variable_t)
#undef RBK_WAIT_PEER

#define RBK_WAIT_ROOT(NAME, TAG)                                                                                     \
  auto nompi_state::NAME(int const root_circuit_index, std::string const& variable_name, int const num_elements)   \
    ->void                                                                                                         \
  {                                                                                                                \
    if (root_circuit_index < 0) return;                                                                            \
    is_waiting_ = true;                                                                                            \
    wait_reason_ = ::bra::wait_reason{::bra::wait_reason::TAG{}, root_circuit_index, variable_name, num_elements}; \
  }
RBK_WAIT_ROOT(do_broadcast_real_variable, broadcast_real_variable_t)
RBK_WAIT_ROOT(do_broadcast_complex_variable, broadcast_complex_variable_t)
RBK_WAIT_ROOT(do_broadcast_int_variable, broadcast_int_variable_t)
#undef RBK_WAIT_ROOT

#define RBK_WAIT_ROOT_NAMED(NAME, TAG)                                                                             \
  auto nompi_state::NAME(int const root_circuit_index, std::string const& variable_name, int const num_elements, \
                         std::string const& other_variable_name)                                                 \
    ->void                                                                                                       \
  {                                                                                                              \
    if (root_circuit_index < 0) return;                                                                          \
    is_waiting_ = true;                                                                                          \
    wait_reason_ = ::bra::wait_reason{::bra::wait_reason::TAG{}, root_circuit_index, variable_name, num_elements,  \
                                      other_variable_name};                                                      \
  }
RBK_WAIT_ROOT_NAMED(do_gather_real_variable, gather_real_variable_t)
RBK_WAIT_ROOT_NAMED(do_gather_complex_variable, gather_complex_variable_t)
RBK_WAIT_ROOT_NAMED(do_gather_int_variable, gather_int_variable_t)
RBK_WAIT_ROOT_NAMED(do_scatter_real_variable, scatter_real_variable_t)
RBK_WAIT_ROOT_NAMED(do_scatter_complex_variable, scatter_complex_variable_t)
RBK_WAIT_ROOT_NAMED(do_scatter_int_variable, scatter_int_variable_t)
#undef RBK_WAIT_ROOT_NAMED

// INNERPROD / FIDELITY with another circuit (its index) or with ALL.
void nompi_state::do_inner_product(std::string const& remote_circuit_index_or_all)
{
  if (std::isdigit(static_cast<unsigned char>(remote_circuit_index_or_all.front()))) {
    auto const other = boost::lexical_cast<int>(remote_circuit_index_or_all);
    if (other < 0 || other == circuit_index_) return;
    is_waiting_ = true;
    wait_reason_ = ::bra::wait_reason{::bra::wait_reason::inner_product_t{}, other};
  } else if (boost::algorithm::to_upper_copy(remote_circuit_index_or_all) == "ALL") {
    is_waiting_ = true;
    wait_reason_ = ::bra::wait_reason{::bra::wait_reason::inner_product_all_t{}};
  }
}

void nompi_state::do_inner_product(std::string const& remote_circuit_index_or_all,
                                   std::string const& operator_literal_or_variable_name,
                                   std::vector<qubit_type> const& operated_qubits)
{
  if (std::isdigit(static_cast<unsigned char>(remote_circuit_index_or_all.front()))) {
    auto const other = boost::lexical_cast<int>(remote_circuit_index_or_all);
    if (other < 0 || other == circuit_index_) return;
    is_waiting_ = true;
    wait_reason_ = ::bra::wait_reason{::bra::wait_reason::inner_product_op_t{}, other, operator_literal_or_variable_name,
                                      operated_qubits};
  } else if (boost::algorithm::to_upper_copy(remote_circuit_index_or_all) == "ALL") {
    is_waiting_ = true;
    wait_reason_ = ::bra::wait_reason{::bra::wait_reason::inner_product_all_op_t{}, operator_literal_or_variable_name,
                                      operated_qubits};
  }
}

void nompi_state::do_fidelity(std::string const& remote_circuit_index_or_all)
{
  if (std::isdigit(static_cast<unsigned char>(remote_circuit_index_or_all.front()))) {
    auto const other = boost::lexical_cast<int>(remote_circuit_index_or_all);
    if (other < 0 || other == circuit_index_) return;
    is_waiting_ = true;
    wait_reason_ = ::bra::wait_reason{::bra::wait_reason::fidelity_t{}, other};
  } else if (boost::algorithm::to_upper_copy(remote_circuit_index_or_all) == "ALL") {
    is_waiting_ = true;
    wait_reason_ = ::bra::wait_reason{::bra::wait_reason::fidelity_all_t{}};
  }
}

void nompi_state::do_fidelity(std::string const& remote_circuit_index_or_all,
                              std::string const& operator_literal_or_variable_name,
                              std::vector<qubit_type> const& operated_qubits)
{
  if (std::isdigit(static_cast<unsigned char>(remote_circuit_index_or_all.front()))) {
    auto const other = boost::lexical_cast<int>(remote_circuit_index_or_all);
    if (other < 0 || other == circuit_index_) return;
    is_waiting_ = true;
    wait_reason_ = ::bra::wait_reason{::bra::wait_reason::fidelity_op_t{}, other, operator_literal_or_variable_name,
                                      operated_qubits};
  } else if (boost::algorithm::to_upper_copy(remote_circuit_index_or_all) == "ALL") {
    is_waiting_ = true;
    wait_reason_ = ::bra::wait_reason{::bra::wait_reason::fidelity_all_op_t{}, operator_literal_or_variable_name,
                                      operated_qubits};
  }
}

// ---- gates ------------------------------------------------------------------------

void nompi_state::do_i_gate(qubit_type const) { }
void nompi_state::do_ic_gate(control_qubit_type const) { }
void nompi_state::do_ii_gate(qubit_type const, qubit_type const) { }
void nompi_state::do_in_gate(std::vector<qubit_type> const&) { }
void nompi_state::do_controlled_i_gate(qubit_type const, control_qubit_type const) { }
void nompi_state::do_controlled_ic_gate(control_qubit_type const, control_qubit_type const) { }
void nompi_state::do_multi_controlled_in_gate(std::vector<qubit_type> const&, std::vector<control_qubit_type> const&) { }
void nompi_state::do_multi_controlled_ic_gate(std::vector<control_qubit_type> const&) { }

void nompi_state::do_hadamard(qubit_type const qubit) { check(rbk_hadamard(handle_, bit(qubit), nullptr, 0)); }
void nompi_state::do_not_(qubit_type const qubit) { check(rbk_pauli_x(handle_, bit(qubit), nullptr, 0)); }
void nompi_state::do_pauli_x(qubit_type const qubit) { check(rbk_pauli_x(handle_, bit(qubit), nullptr, 0)); }
void nompi_state::do_pauli_y(qubit_type const qubit) { check(rbk_pauli_y(handle_, bit(qubit), nullptr, 0)); }
void nompi_state::do_pauli_z(control_qubit_type const control_qubit)
{
  std::uint32_t const q = bit(control_qubit);
  check(rbk_pauli_z(handle_, &q, 1));
}

namespace {
// A product of one Pauli letter on each target, under controls.
void pauli_product(rbk_state* const s, char const letter, std::vector<std::uint32_t> const& targets,
                   std::vector<std::uint32_t> const& controls = {})
{
  const std::string letters(targets.size(), letter);
  check(rbk_pauli_string(s, letters.c_str(), targets.data(), size_of(targets), controls.data(), size_of(controls)));
}
void exponential_product(rbk_state* const s, double const phase, char const letter, std::vector<std::uint32_t> const& targets,
                         std::vector<std::uint32_t> const& controls = {})
{
  const std::string letters(targets.size(), letter);
  check(rbk_exponential_pauli_string(s, phase, letters.c_str(), targets.data(), size_of(targets), controls.data(),
                                     size_of(controls)));
}
}  // namespace

void nompi_state::do_pauli_xx(qubit_type const q1, qubit_type const q2) { pauli_product(handle_, 'X', {bit(q1), bit(q2)}); }
void nompi_state::do_pauli_xn(std::vector<qubit_type> const& qubits) { pauli_product(handle_, 'X', bits(qubits)); }
void nompi_state::do_pauli_yy(qubit_type const q1, qubit_type const q2) { pauli_product(handle_, 'Y', {bit(q1), bit(q2)}); }
void nompi_state::do_pauli_yn(std::vector<qubit_type> const& qubits) { pauli_product(handle_, 'Y', bits(qubits)); }
void nompi_state::do_pauli_zz(qubit_type const q1, qubit_type const q2) { pauli_product(handle_, 'Z', {bit(q1), bit(q2)}); }
void nompi_state::do_pauli_zn(std::vector<qubit_type> const& qubits) { pauli_product(handle_, 'Z', bits(qubits)); }
void nompi_state::do_swap(qubit_type const q1, qubit_type const q2) { check(rbk_swap(handle_, bit(q1), bit(q2), nullptr, 0)); }

void nompi_state::do_sqrt_pauli_x(qubit_type const q) { check(rbk_sqrt_pauli_x(handle_, 0, bit(q), nullptr, 0)); }
void nompi_state::do_adj_sqrt_pauli_x(qubit_type const q) { check(rbk_sqrt_pauli_x(handle_, 1, bit(q), nullptr, 0)); }
void nompi_state::do_sqrt_pauli_y(qubit_type const q) { check(rbk_sqrt_pauli_y(handle_, 0, bit(q), nullptr, 0)); }
void nompi_state::do_adj_sqrt_pauli_y(qubit_type const q) { check(rbk_sqrt_pauli_y(handle_, 1, bit(q), nullptr, 0)); }
void nompi_state::do_sqrt_pauli_z(control_qubit_type const c)
{
  std::uint32_t const q = bit(c);
  check(rbk_sqrt_pauli_z(handle_, 0, &q, 1, nullptr, 0));
}
void nompi_state::do_adj_sqrt_pauli_z(control_qubit_type const c)
{
  std::uint32_t const q = bit(c);
  check(rbk_sqrt_pauli_z(handle_, 1, &q, 1, nullptr, 0));
}
void nompi_state::do_sqrt_pauli_zz(qubit_type const q1, qubit_type const q2)
{
  std::uint32_t const t[2] = {bit(q1), bit(q2)};
  check(rbk_sqrt_pauli_z(handle_, 0, t, 2, nullptr, 0));
}
void nompi_state::do_adj_sqrt_pauli_zz(qubit_type const q1, qubit_type const q2)
{
  std::uint32_t const t[2] = {bit(q1), bit(q2)};
  check(rbk_sqrt_pauli_z(handle_, 1, t, 2, nullptr, 0));
}
void nompi_state::do_sqrt_pauli_zn(std::vector<qubit_type> const& qubits)
{
  auto const t = bits(qubits);
  check(rbk_sqrt_pauli_z(handle_, 0, t.data(), size_of(t), nullptr, 0));
}
void nompi_state::do_adj_sqrt_pauli_zn(std::vector<qubit_type> const& qubits)
{
  auto const t = bits(qubits);
  check(rbk_sqrt_pauli_z(handle_, 1, t.data(), size_of(t), nullptr, 0));
}

void nompi_state::do_u1(real_type const phase, control_qubit_type const c)
{
  std::uint32_t const q = bit(c);
  check(rbk_phase_shift(handle_, phase, &q, 1));
}
void nompi_state::do_adj_u1(real_type const phase, control_qubit_type const c)
{
  std::uint32_t const q = bit(c);
  check(rbk_phase_shift(handle_, -phase, &q, 1));
}
// U2(phi, lambda)^dagger = U3(-pi/2, -lambda, -phi); U3(theta, phi, lambda)^dagger = U3(-theta, -lambda, -phi).
void nompi_state::do_u2(real_type const phase1, real_type const phase2, qubit_type const q)
{
  check(rbk_phase_shift2(handle_, phase1, phase2, bit(q), nullptr, 0));
}
void nompi_state::do_adj_u2(real_type const phase1, real_type const phase2, qubit_type const q)
{
  check(rbk_phase_shift3(handle_, -kHalfPi, -phase2, -phase1, bit(q), nullptr, 0));
}
void nompi_state::do_u3(real_type const phase1, real_type const phase2, real_type const phase3, qubit_type const q)
{
  check(rbk_phase_shift3(handle_, phase1, phase2, phase3, bit(q), nullptr, 0));
}
void nompi_state::do_adj_u3(real_type const phase1, real_type const phase2, real_type const phase3, qubit_type const q)
{
  check(rbk_phase_shift3(handle_, -phase1, -phase3, -phase2, bit(q), nullptr, 0));
}
void nompi_state::do_phase_shift(complex_type const& coefficient, control_qubit_type const c)
{
  std::uint32_t const q = bit(c);
  check(rbk_phase_shift_coeff(handle_, coefficient.real(), coefficient.imag(), &q, 1));
}
void nompi_state::do_adj_phase_shift(complex_type const& coefficient, control_qubit_type const c)
{
  std::uint32_t const q = bit(c);
  check(rbk_phase_shift_coeff(handle_, coefficient.real(), -coefficient.imag(), &q, 1));
}
void nompi_state::do_x_rotation_half_pi(qubit_type const q) { check(rbk_x_rotation_half_pi(handle_, 0, bit(q), nullptr, 0)); }
void nompi_state::do_adj_x_rotation_half_pi(qubit_type const q) { check(rbk_x_rotation_half_pi(handle_, 1, bit(q), nullptr, 0)); }
void nompi_state::do_y_rotation_half_pi(qubit_type const q) { check(rbk_y_rotation_half_pi(handle_, 0, bit(q), nullptr, 0)); }
void nompi_state::do_adj_y_rotation_half_pi(qubit_type const q) { check(rbk_y_rotation_half_pi(handle_, 1, bit(q), nullptr, 0)); }

// exp(i phase P) and its adjoint exp(-i phase P).
void nompi_state::do_exponential_pauli_x(real_type const phase, qubit_type const q)
{
  check(rbk_exponential_pauli_x(handle_, phase, bit(q), nullptr, 0));
}
void nompi_state::do_adj_exponential_pauli_x(real_type const phase, qubit_type const q)
{
  check(rbk_exponential_pauli_x(handle_, -phase, bit(q), nullptr, 0));
}
void nompi_state::do_exponential_pauli_y(real_type const phase, qubit_type const q)
{
  check(rbk_exponential_pauli_y(handle_, phase, bit(q), nullptr, 0));
}
void nompi_state::do_adj_exponential_pauli_y(real_type const phase, qubit_type const q)
{
  check(rbk_exponential_pauli_y(handle_, -phase, bit(q), nullptr, 0));
}
void nompi_state::do_exponential_pauli_z(real_type const phase, qubit_type const q)
{
  check(rbk_exponential_pauli_z(handle_, phase, bit(q), nullptr, 0));
}
void nompi_state::do_adj_exponential_pauli_z(real_type const phase, qubit_type const q)
{
  check(rbk_exponential_pauli_z(handle_, -phase, bit(q), nullptr, 0));
}
void nompi_state::do_exponential_pauli_xx(real_type const phase, qubit_type const q1, qubit_type const q2)
{
  exponential_product(handle_, phase, 'X', {bit(q1), bit(q2)});
}
void nompi_state::do_adj_exponential_pauli_xx(real_type const phase, qubit_type const q1, qubit_type const q2)
{
  exponential_product(handle_, -phase, 'X', {bit(q1), bit(q2)});
}
void nompi_state::do_exponential_pauli_xn(real_type const phase, std::vector<qubit_type> const& qubits)
{
  exponential_product(handle_, phase, 'X', bits(qubits));
}
void nompi_state::do_adj_exponential_pauli_xn(real_type const phase, std::vector<qubit_type> const& qubits)
{
  exponential_product(handle_, -phase, 'X', bits(qubits));
}
void nompi_state::do_exponential_pauli_yy(real_type const phase, qubit_type const q1, qubit_type const q2)
{
  exponential_product(handle_, phase, 'Y', {bit(q1), bit(q2)});
}
void nompi_state::do_adj_exponential_pauli_yy(real_type const phase, qubit_type const q1, qubit_type const q2)
{
  exponential_product(handle_, -phase, 'Y', {bit(q1), bit(q2)});
}
void nompi_state::do_exponential_pauli_yn(real_type const phase, std::vector<qubit_type> const& qubits)
{
  exponential_product(handle_, phase, 'Y', bits(qubits));
}
void nompi_state::do_adj_exponential_pauli_yn(real_type const phase, std::vector<qubit_type> const& qubits)
{
  exponential_product(handle_, -phase, 'Y', bits(qubits));
}
void nompi_state::do_exponential_pauli_zz(real_type const phase, qubit_type const q1, qubit_type const q2)
{
  exponential_product(handle_, phase, 'Z', {bit(q1), bit(q2)});
}
void nompi_state::do_adj_exponential_pauli_zz(real_type const phase, qubit_type const q1, qubit_type const q2)
{
  exponential_product(handle_, -phase, 'Z', {bit(q1), bit(q2)});
}
void nompi_state::do_exponential_pauli_zn(real_type const phase, std::vector<qubit_type> const& qubits)
{
  exponential_product(handle_, phase, 'Z', bits(qubits));
}
void nompi_state::do_adj_exponential_pauli_zn(real_type const phase, std::vector<qubit_type> const& qubits)
{
  exponential_product(handle_, -phase, 'Z', bits(qubits));
}
void nompi_state::do_exponential_swap(real_type const phase, qubit_type const q1, qubit_type const q2)
{
  check(rbk_exponential_swap(handle_, phase, bit(q1), bit(q2), nullptr, 0));
}
void nompi_state::do_adj_exponential_swap(real_type const phase, qubit_type const q1, qubit_type const q2)
{
  check(rbk_exponential_swap(handle_, -phase, bit(q1), bit(q2), nullptr, 0));
}
void nompi_state::do_toffoli(qubit_type const target, control_qubit_type const c1, control_qubit_type const c2)
{
  auto const cs = bits({c1, c2});
  check(rbk_pauli_x(handle_, bit(target), cs.data(), 2));
}

// ---- controlled gates ----------------------------------------------------------------

void nompi_state::do_controlled_hadamard(qubit_type const t, control_qubit_type const c)
{
  auto const cs = bits({c});
  check(rbk_hadamard(handle_, bit(t), cs.data(), 1));
}
void nompi_state::do_multi_controlled_hadamard(qubit_type const t, std::vector<control_qubit_type> const& controls)
{
  auto const cs = bits(controls);
  check(rbk_hadamard(handle_, bit(t), cs.data(), size_of(cs)));
}
void nompi_state::do_controlled_not(qubit_type const t, control_qubit_type const c)
{
  auto const cs = bits({c});
  check(rbk_pauli_x(handle_, bit(t), cs.data(), 1));
}
void nompi_state::do_multi_controlled_not(qubit_type const t, std::vector<control_qubit_type> const& controls)
{
  auto const cs = bits(controls);
  check(rbk_pauli_x(handle_, bit(t), cs.data(), size_of(cs)));
}
void nompi_state::do_controlled_pauli_x(qubit_type const t, control_qubit_type const c)
{
  auto const cs = bits({c});
  check(rbk_pauli_x(handle_, bit(t), cs.data(), 1));
}
void nompi_state::do_multi_controlled_pauli_xn(std::vector<qubit_type> const& targets, std::vector<control_qubit_type> const& controls)
{
  pauli_product(handle_, 'X', bits(targets), bits(controls));
}
void nompi_state::do_controlled_pauli_y(qubit_type const t, control_qubit_type const c)
{
  auto const cs = bits({c});
  check(rbk_pauli_y(handle_, bit(t), cs.data(), 1));
}
void nompi_state::do_multi_controlled_pauli_yn(std::vector<qubit_type> const& targets, std::vector<control_qubit_type> const& controls)
{
  pauli_product(handle_, 'Y', bits(targets), bits(controls));
}
void nompi_state::do_controlled_pauli_z(control_qubit_type const c1, control_qubit_type const c2)
{
  auto const qs = bits({c1, c2});
  check(rbk_pauli_z(handle_, qs.data(), 2));
}
void nompi_state::do_multi_controlled_pauli_z(std::vector<control_qubit_type> const& controls)
{
  auto const qs = bits(controls);
  check(rbk_pauli_z(handle_, qs.data(), size_of(qs)));
}
void nompi_state::do_multi_controlled_pauli_zn(std::vector<qubit_type> const& targets, std::vector<control_qubit_type> const& controls)
{
  pauli_product(handle_, 'Z', bits(targets), bits(controls));
}
void nompi_state::do_multi_controlled_swap(qubit_type const t1, qubit_type const t2, std::vector<control_qubit_type> const& controls)
{
  auto const cs = bits(controls);
  check(rbk_swap(handle_, bit(t1), bit(t2), cs.data(), size_of(cs)));
}

#define RBK_CTRL_1Q(NAME, CALL, ADJ)                                                                        \
  void nompi_state::NAME(qubit_type const t, control_qubit_type const c)                                    \
  {                                                                                                         \
    auto const cs = bits({c});                                                                              \
    check(CALL(handle_, ADJ, bit(t), cs.data(), 1));                                                        \
  }
#define RBK_MCTRL_1Q(NAME, CALL, ADJ)                                                                       \
  void nompi_state::NAME(qubit_type const t, std::vector<control_qubit_type> const& controls)               \
  {                                                                                                         \
    auto const cs = bits(controls);                                                                         \
    check(CALL(handle_, ADJ, bit(t), cs.data(), size_of(cs)));                                              \
  }
RBK_CTRL_1Q(do_controlled_sqrt_pauli_x, rbk_sqrt_pauli_x, 0)
RBK_CTRL_1Q(do_adj_controlled_sqrt_pauli_x, rbk_sqrt_pauli_x, 1)
RBK_MCTRL_1Q(do_multi_controlled_sqrt_pauli_x, rbk_sqrt_pauli_x, 0)
RBK_MCTRL_1Q(do_adj_multi_controlled_sqrt_pauli_x, rbk_sqrt_pauli_x, 1)
RBK_CTRL_1Q(do_controlled_sqrt_pauli_y, rbk_sqrt_pauli_y, 0)
RBK_CTRL_1Q(do_adj_controlled_sqrt_pauli_y, rbk_sqrt_pauli_y, 1)
RBK_MCTRL_1Q(do_multi_controlled_sqrt_pauli_y, rbk_sqrt_pauli_y, 0)
RBK_MCTRL_1Q(do_adj_multi_controlled_sqrt_pauli_y, rbk_sqrt_pauli_y, 1)
RBK_CTRL_1Q(do_controlled_x_rotation_half_pi, rbk_x_rotation_half_pi, 0)
RBK_CTRL_1Q(do_adj_controlled_x_rotation_half_pi, rbk_x_rotation_half_pi, 1)
RBK_MCTRL_1Q(do_multi_controlled_x_rotation_half_pi, rbk_x_rotation_half_pi, 0)
RBK_MCTRL_1Q(do_adj_multi_controlled_x_rotation_half_pi, rbk_x_rotation_half_pi, 1)
RBK_CTRL_1Q(do_controlled_y_rotation_half_pi, rbk_y_rotation_half_pi, 0)
RBK_CTRL_1Q(do_adj_controlled_y_rotation_half_pi, rbk_y_rotation_half_pi, 1)
RBK_MCTRL_1Q(do_multi_controlled_y_rotation_half_pi, rbk_y_rotation_half_pi, 0)
RBK_MCTRL_1Q(do_adj_multi_controlled_y_rotation_half_pi, rbk_y_rotation_half_pi, 1)
#undef RBK_CTRL_1Q
#undef RBK_MCTRL_1Q

// sqrt(Z) is diagonal: i on the amplitudes whose listed qubits are all one, so
// the first listed qubit serves as the target and the rest as controls.
namespace {
void sqrt_z_on(rbk_state* const s, int const adjoint, std::vector<std::uint32_t> const& qubits)
{
  check(rbk_sqrt_pauli_z(s, adjoint, qubits.data(), 1, qubits.data() + 1, size_of(qubits) - 1));
}
}  // namespace
void nompi_state::do_controlled_sqrt_pauli_z(control_qubit_type const c1, control_qubit_type const c2)
{
  sqrt_z_on(handle_, 0, bits({c1, c2}));
}
void nompi_state::do_adj_controlled_sqrt_pauli_z(control_qubit_type const c1, control_qubit_type const c2)
{
  sqrt_z_on(handle_, 1, bits({c1, c2}));
}
void nompi_state::do_multi_controlled_sqrt_pauli_z(std::vector<control_qubit_type> const& controls)
{
  sqrt_z_on(handle_, 0, bits(controls));
}
void nompi_state::do_adj_multi_controlled_sqrt_pauli_z(std::vector<control_qubit_type> const& controls)
{
  sqrt_z_on(handle_, 1, bits(controls));
}
void nompi_state::do_multi_controlled_sqrt_pauli_zn(std::vector<qubit_type> const& targets, std::vector<control_qubit_type> const& controls)
{
  auto const t = bits(targets);
  auto const cs = bits(controls);
  check(rbk_sqrt_pauli_z(handle_, 0, t.data(), size_of(t), cs.data(), size_of(cs)));
}
void nompi_state::do_adj_multi_controlled_sqrt_pauli_zn(std::vector<qubit_type> const& targets,
                                                        std::vector<control_qubit_type> const& controls)
{
  auto const t = bits(targets);
  auto const cs = bits(controls);
  check(rbk_sqrt_pauli_z(handle_, 1, t.data(), size_of(t), cs.data(), size_of(cs)));
}

void nompi_state::do_controlled_phase_shift(complex_type const& coefficient, control_qubit_type const c1, control_qubit_type const c2)
{
  auto const qs = bits({c1, c2});
  check(rbk_phase_shift_coeff(handle_, coefficient.real(), coefficient.imag(), qs.data(), 2));
}
void nompi_state::do_adj_controlled_phase_shift(complex_type const& coefficient, control_qubit_type const c1,
                                                control_qubit_type const c2)
{
  auto const qs = bits({c1, c2});
  check(rbk_phase_shift_coeff(handle_, coefficient.real(), -coefficient.imag(), qs.data(), 2));
}
void nompi_state::do_multi_controlled_phase_shift(complex_type const& coefficient, std::vector<control_qubit_type> const& controls)
{
  auto const qs = bits(controls);
  check(rbk_phase_shift_coeff(handle_, coefficient.real(), coefficient.imag(), qs.data(), size_of(qs)));
}
void nompi_state::do_adj_multi_controlled_phase_shift(complex_type const& coefficient,
                                                      std::vector<control_qubit_type> const& controls)
{
  auto const qs = bits(controls);
  check(rbk_phase_shift_coeff(handle_, coefficient.real(), -coefficient.imag(), qs.data(), size_of(qs)));
}
void nompi_state::do_controlled_u1(real_type const phase, control_qubit_type const c1, control_qubit_type const c2)
{
  auto const qs = bits({c1, c2});
  check(rbk_phase_shift(handle_, phase, qs.data(), 2));
}
void nompi_state::do_adj_controlled_u1(real_type const phase, control_qubit_type const c1, control_qubit_type const c2)
{
  auto const qs = bits({c1, c2});
  check(rbk_phase_shift(handle_, -phase, qs.data(), 2));
}
void nompi_state::do_multi_controlled_u1(real_type const phase, std::vector<control_qubit_type> const& controls)
{
  auto const qs = bits(controls);
  check(rbk_phase_shift(handle_, phase, qs.data(), size_of(qs)));
}
void nompi_state::do_adj_multi_controlled_u1(real_type const phase, std::vector<control_qubit_type> const& controls)
{
  auto const qs = bits(controls);
  check(rbk_phase_shift(handle_, -phase, qs.data(), size_of(qs)));
}
void nompi_state::do_controlled_u2(real_type const phase1, real_type const phase2, qubit_type const t, control_qubit_type const c)
{
  auto const cs = bits({c});
  check(rbk_phase_shift2(handle_, phase1, phase2, bit(t), cs.data(), 1));
}
void nompi_state::do_adj_controlled_u2(real_type const phase1, real_type const phase2, qubit_type const t,
                                       control_qubit_type const c)
{
  auto const cs = bits({c});
  check(rbk_phase_shift3(handle_, -kHalfPi, -phase2, -phase1, bit(t), cs.data(), 1));
}
void nompi_state::do_multi_controlled_u2(real_type const phase1, real_type const phase2, qubit_type const t,
                                         std::vector<control_qubit_type> const& controls)
{
  auto const cs = bits(controls);
  check(rbk_phase_shift2(handle_, phase1, phase2, bit(t), cs.data(), size_of(cs)));
}
void nompi_state::do_adj_multi_controlled_u2(real_type const phase1, real_type const phase2, qubit_type const t,
                                             std::vector<control_qubit_type> const& controls)
{
  auto const cs = bits(controls);
  check(rbk_phase_shift3(handle_, -kHalfPi, -phase2, -phase1, bit(t), cs.data(), size_of(cs)));
}
void nompi_state::do_controlled_u3(real_type const phase1, real_type const phase2, real_type const phase3, qubit_type const t,
                                   control_qubit_type const c)
{
  auto const cs = bits({c});
  check(rbk_phase_shift3(handle_, phase1, phase2, phase3, bit(t), cs.data(), 1));
}
void nompi_state::do_adj_controlled_u3(real_type const phase1, real_type const phase2, real_type const phase3,
                                       qubit_type const t, control_qubit_type const c)
{
  auto const cs = bits({c});
  check(rbk_phase_shift3(handle_, -phase1, -phase3, -phase2, bit(t), cs.data(), 1));
}
void nompi_state::do_multi_controlled_u3(real_type const phase1, real_type const phase2, real_type const phase3,
                                         qubit_type const t, std::vector<control_qubit_type> const& controls)
{
  auto const cs = bits(controls);
  check(rbk_phase_shift3(handle_, phase1, phase2, phase3, bit(t), cs.data(), size_of(cs)));
}
void nompi_state::do_adj_multi_controlled_u3(real_type const phase1, real_type const phase2, real_type const phase3,
                                             qubit_type const t, std::vector<control_qubit_type> const& controls)
{
  auto const cs = bits(controls);
  check(rbk_phase_shift3(handle_, -phase1, -phase3, -phase2, bit(t), cs.data(), size_of(cs)));
}

#define RBK_CTRL_EXP(NAME, CALL, SIGN)                                                                   \
  void nompi_state::NAME(real_type const phase, qubit_type const t, control_qubit_type const c)          \
  {                                                                                                      \
    auto const cs = bits({c});                                                                           \
    check(CALL(handle_, SIGN phase, bit(t), cs.data(), 1));                                              \
  }
RBK_CTRL_EXP(do_controlled_exponential_pauli_x, rbk_exponential_pauli_x, +)
RBK_CTRL_EXP(do_adj_controlled_exponential_pauli_x, rbk_exponential_pauli_x, -)
RBK_CTRL_EXP(do_controlled_exponential_pauli_y, rbk_exponential_pauli_y, +)
RBK_CTRL_EXP(do_adj_controlled_exponential_pauli_y, rbk_exponential_pauli_y, -)
RBK_CTRL_EXP(do_controlled_exponential_pauli_z, rbk_exponential_pauli_z, +)
RBK_CTRL_EXP(do_adj_controlled_exponential_pauli_z, rbk_exponential_pauli_z, -)
#undef RBK_CTRL_EXP

void nompi_state::do_multi_controlled_exponential_pauli_xn(real_type const phase, std::vector<qubit_type> const& targets,
                                                           std::vector<control_qubit_type> const& controls)
{
  exponential_product(handle_, phase, 'X', bits(targets), bits(controls));
}
void nompi_state::do_adj_multi_controlled_exponential_pauli_xn(real_type const phase, std::vector<qubit_type> const& targets,
                                                               std::vector<control_qubit_type> const& controls)
{
  exponential_product(handle_, -phase, 'X', bits(targets), bits(controls));
}
void nompi_state::do_multi_controlled_exponential_pauli_yn(real_type const phase, std::vector<qubit_type> const& targets,
                                                           std::vector<control_qubit_type> const& controls)
{
  exponential_product(handle_, phase, 'Y', bits(targets), bits(controls));
}
void nompi_state::do_adj_multi_controlled_exponential_pauli_yn(real_type const phase, std::vector<qubit_type> const& targets,
                                                               std::vector<control_qubit_type> const& controls)
{
  exponential_product(handle_, -phase, 'Y', bits(targets), bits(controls));
}
void nompi_state::do_multi_controlled_exponential_pauli_z(real_type const phase, qubit_type const t,
                                                          std::vector<control_qubit_type> const& controls)
{
  auto const cs = bits(controls);
  check(rbk_exponential_pauli_z(handle_, phase, bit(t), cs.data(), size_of(cs)));
}
void nompi_state::do_adj_multi_controlled_exponential_pauli_z(real_type const phase, qubit_type const t,
                                                              std::vector<control_qubit_type> const& controls)
{
  auto const cs = bits(controls);
  check(rbk_exponential_pauli_z(handle_, -phase, bit(t), cs.data(), size_of(cs)));
}
void nompi_state::do_multi_controlled_exponential_pauli_zn(real_type const phase, std::vector<qubit_type> const& targets,
                                                           std::vector<control_qubit_type> const& controls)
{
  exponential_product(handle_, phase, 'Z', bits(targets), bits(controls));
}
void nompi_state::do_adj_multi_controlled_exponential_pauli_zn(real_type const phase, std::vector<qubit_type> const& targets,
                                                               std::vector<control_qubit_type> const& controls)
{
  exponential_product(handle_, -phase, 'Z', bits(targets), bits(controls));
}
void nompi_state::do_multi_controlled_exponential_swap(real_type const phase, qubit_type const t1, qubit_type const t2,
                                                       std::vector<control_qubit_type> const& controls)
{
  auto const cs = bits(controls);
  check(rbk_exponential_swap(handle_, phase, bit(t1), bit(t2), cs.data(), size_of(cs)));
}
void nompi_state::do_adj_multi_controlled_exponential_swap(real_type const phase, qubit_type const t1, qubit_type const t2,
                                                           std::vector<control_qubit_type> const& controls)
{
  auto const cs = bits(controls);
  check(rbk_exponential_swap(handle_, -phase, bit(t1), bit(t2), cs.data(), size_of(cs)));
}

// ---- fusion, reads, measurements ------------------------------------------------------

void nompi_state::do_begin_fusion() { check(rbk_begin_fusion(handle_)); }
void nompi_state::do_end_fusion() { check(rbk_end_fusion(handle_)); }
void nompi_state::do_clear(qubit_type const q) { check(rbk_clear(handle_, bit(q))); }
void nompi_state::do_set(qubit_type const q) { check(rbk_set(handle_, bit(q))); }

// SHORBOX: bra::state::shor_box passes the exponent register as the top
// qubits and the rest as the work register, the layout the engine's shor box uses.
void nompi_state::do_shor_box(state_integer_type const divisor, state_integer_type const base,
                              std::vector<qubit_type> const& exponent_qubits,
                              std::vector<qubit_type> const& modular_exponentiation_qubits)
{
  auto const n = static_cast<std::uint32_t>(total_num_qubits_);
  auto const nx = static_cast<std::uint32_t>(exponent_qubits.size());
  for (std::uint32_t k = 0; k < nx; ++k)
    if (bit(exponent_qubits[k]) != n - nx + k) throw std::runtime_error("SHORBOX: exponent register not on the top qubits");
  for (std::uint32_t k = 0; k < modular_exponentiation_qubits.size(); ++k)
    if (bit(modular_exponentiation_qubits[k]) != k) throw std::runtime_error("SHORBOX: work register not on the low qubits");
  check(rbk_shor_box(handle_, nx, divisor, base));
}

// DO MEASUREMENT: all spins in ket's convention; bra::state prints them.
void nompi_state::do_expectation_values()
{
  auto const n = static_cast<std::size_t>(total_num_qubits_);
  std::vector<double> out(3 * n);
  check(rbk_spin_expectation_values(handle_, out.data()));
  spins_type spins(n);
  for (std::size_t q = 0; q < n; ++q)
    for (std::size_t k = 0; k < 3; ++k) spins[q][k] = static_cast<real_type>(out[3 * q + k]);
  maybe_expectation_values_ = std::move(spins);
}

// PRINT AMPLITUDES: "bits => re + im i" per amplitude, with the stream's
// default formatting; all amplitudes (newline-separated, newline at the end)
// or the listed ones.
void nompi_state::do_amplitudes(std::vector< ::bra::state_integer_type > const& amplitude_indices)
{
  std::ostringstream oss;
  auto line = [this, &oss](::bra::state_integer_type const index, complex_type const& a) {
    oss << ::bra::state_detail::integer_to_bits_string(index, total_num_qubits_) << " => " << a.real() << " + " << a.imag() << " i";
  };
  if (amplitude_indices.empty()) {
    std::vector<complex_type> all(std::size_t{1} << total_num_qubits_);
    check(rbk_state_download(handle_, all.data(), 0u, all.size()));
    for (std::size_t i = 0; i < all.size(); ++i) {
      if (i) oss << '\n';
      line(i, all[i]);
    }
    oss << '\n';
  } else {
    for (auto const index : amplitude_indices) {
      complex_type a;
      check(rbk_state_download(handle_, &a, index, 1u));
      line(index, a);
      oss << '\n';
    }
  }
  std::cout << oss.str() << std::flush;
}

ket::gate::outcome nompi_state::do_projective_measurement(qubit_type const qubit)
{
  int one = 0;
  check(rbk_projective_measurement_with(handle_, bit(qubit), &draw_upto, &random_number_generator_, &one));
  return one ? ket::gate::outcome::one : ket::gate::outcome::zero;
}

void nompi_state::do_measure()
{
  std::uint64_t outcome = 0;
  check(rbk_measure_with(handle_, &draw_upto, &random_number_generator_, &outcome));
  measured_value_ = static_cast<state_integer_type>(outcome);
}

// GENERATE EVENTS n [seed]: a negative seed draws from the state's generator,
// otherwise from a fresh generator built from the seed (ket::generate_events).
void nompi_state::do_generate_events(int const num_events, int const seed)
{
  std::vector<std::uint64_t> events(static_cast<std::size_t>(num_events > 0 ? num_events : 0));
  if (seed < 0) {
    check(rbk_generate_events_with(handle_, num_events, &draw_upto, &random_number_generator_, events.data()));
  } else {
    random_number_generator_type engine(static_cast<seed_type>(seed));
    check(rbk_generate_events_with(handle_, num_events, &draw_upto, &engine, events.data()));
  }
  generated_events_.assign(events.begin(), events.end());
}

void nompi_state::do_expectation_value(std::string const& operator_literal_or_variable_name,
                                       std::vector<qubit_type> const& operated_qubits)
{
  auto const op = to_pauli_string_space(operator_literal_or_variable_name);
  if (operated_qubits.size() != op.num_qubits())
    throw ::bra::wrong_pauli_string_length_error{operated_qubits.size(), op.num_qubits()};
  std::string strings;
  std::vector<double> coeffs;
  operator_terms(op, operated_qubits, total_num_qubits_, strings, coeffs);
  double r[2];
  check(rbk_expectation_pauli(handle_, static_cast<int>(coeffs.size() / 2), strings.c_str(), coeffs.data(), r));
  result_ = complex_type{r[0], r[1]};
}

// ---- the free functions bra's main calls for waiting states -----------------------------

namespace {
complex_type inner(nompi_state& a, nompi_state& b)
{
  double r[2];
  check(rbk_inner_product(a.handle(), b.handle(), r));
  return complex_type{r[0], r[1]};
}
double fid(nompi_state& a, nompi_state& b)
{
  double r = 0;
  check(rbk_fidelity(a.handle(), b.handle(), &r));
  return r;
}
}  // namespace

// <state2|state1> as ket::ranges::inner_product(state1, state2) gives it; the
// other circuit gets the conjugate.
void inner_product(nompi_state& state1, nompi_state& state2)
{
  auto const r = inner(state1, state2);
  state1.result_ = r;
  state2.result_ = std::conj(r);
}

void inner_product_all(std::vector<nompi_state>& states)
{
  for (auto& s : states) s.result_ = inner(states.front(), s);
}

namespace {
// <state2| H |state1> for the operator on the operated qubits, with bra's checks.
complex_type inner_op(nompi_state& state1, nompi_state& state2, ::bra::pauli_string_space const& op,
                      std::vector< ::bra::qubit_type > const& operated_qubits, unsigned const num_qubits, bool const squared)
{
  std::string strings;
  std::vector<double> coeffs;
  operator_terms(op, operated_qubits, num_qubits, strings, coeffs);
  double r[2] = {0, 0};
  if (squared) {
    check(rbk_fidelity_pauli(state1.handle(), state2.handle(), static_cast<int>(coeffs.size() / 2), strings.c_str(),
                             coeffs.data(), r));
    return complex_type{r[0], 0.0};
  }
  check(rbk_inner_product_pauli(state1.handle(), state2.handle(), static_cast<int>(coeffs.size() / 2), strings.c_str(),
                                coeffs.data(), r));
  return complex_type{r[0], r[1]};
}
}  // namespace

#define RBK_OP_CHECKS(FIRST)                                                                                    \
  auto const num_operated = operated_qubits.size();                                                            \
  if (num_operated > (FIRST).total_num_qubits_)                                                                \
    throw ::bra::too_many_operated_qubits_error{num_operated, (FIRST).total_num_qubits_};                      \
  auto const op = (FIRST).to_pauli_string_space(operator_literal_or_variable_name);                           \
  if (num_operated != op.num_qubits()) throw ::bra::wrong_pauli_string_length_error{num_operated, op.num_qubits()};

void inner_product_op(nompi_state& state1, nompi_state& state2, std::string const& operator_literal_or_variable_name,
                      std::vector< ::bra::qubit_type > const& operated_qubits)
{
  RBK_OP_CHECKS(state1)
  auto const r = inner_op(state1, state2, op, operated_qubits, state1.total_num_qubits_, false);
  state1.result_ = r;
  state2.result_ = std::conj(r);
}

void inner_product_all_op(std::vector<nompi_state>& states, std::string const& operator_literal_or_variable_name,
                          std::vector< ::bra::qubit_type > const& operated_qubits)
{
  RBK_OP_CHECKS(states.front())
  for (auto& s : states) s.result_ = inner_op(states.front(), s, op, operated_qubits, states.front().total_num_qubits_, false);
}

void fidelity(nompi_state& state1, nompi_state& state2)
{
  auto const r = fid(state1, state2);
  state1.result_ = r;
  state2.result_ = r;
}

void fidelity_all(std::vector<nompi_state>& states)
{
  for (auto& s : states) s.result_ = fid(states.front(), s);
}

void fidelity_op(nompi_state& state1, nompi_state& state2, std::string const& operator_literal_or_variable_name,
                 std::vector< ::bra::qubit_type > const& operated_qubits)
{
  RBK_OP_CHECKS(state1)
  auto const r = inner_op(state1, state2, op, operated_qubits, state1.total_num_qubits_, true);
  state1.result_ = r;
  state2.result_ = std::conj(r);
}

void fidelity_all_op(std::vector<nompi_state>& states, std::string const& operator_literal_or_variable_name,
                     std::vector< ::bra::qubit_type > const& operated_qubits)
{
  RBK_OP_CHECKS(states.front())
  for (auto& s : states) s.result_ = inner_op(states.front(), s, op, operated_qubits, states.front().total_num_qubits_, true);
}
#undef RBK_OP_CHECKS

// Classical variables between circuits.  A variable's elements are contiguous
// from the element to_*_variable names; num_elements of them are copied.
#define RBK_VARIABLE_TRANSFERS(KIND)                                                                               \
  void send_##KIND##_variable(nompi_state const& source_state, std::string const& source_variable_name,           \
                              nompi_state& destination_state, std::string const& destination_variable_name,       \
                              int const num_elements)                                                             \
  {                                                                                                               \
    auto const* from = std::addressof(source_state.to_##KIND##_variable(source_variable_name));                   \
    auto* to = std::addressof(destination_state.to_##KIND##_variable(destination_variable_name));                 \
    std::copy(from, from + num_elements, to);                                                                     \
  }                                                                                                               \
  void broadcast_##KIND##_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names, \
                                   int const root_circuit_index, int const num_elements)                          \
  {                                                                                                               \
    auto const* from = std::addressof(states[root_circuit_index].to_##KIND##_variable(variable_names[root_circuit_index])); \
    for (int c = 0; c < static_cast<int>(states.size()); ++c) {                                                   \
      if (c == root_circuit_index) continue;                                                                      \
      std::copy(from, from + num_elements, std::addressof(states[c].to_##KIND##_variable(variable_names[c])));     \
    }                                                                                                             \
  }                                                                                                               \
  void gather_##KIND##_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names,  \
                                std::string const& destination_variable_name, int const root_circuit_index,       \
                                int const num_elements)                                                           \
  {                                                                                                               \
    bool const named = !destination_variable_name.empty();                                                        \
    auto* to = std::addressof(states[root_circuit_index].to_##KIND##_variable(                                    \
      named ? destination_variable_name : variable_names[root_circuit_index]));                                   \
    for (int c = 0; c < static_cast<int>(states.size()); ++c) {                                                   \
      if (c == root_circuit_index && !named) continue;                                                            \
      auto const* from = std::addressof(states[c].to_##KIND##_variable(variable_names[c]));                        \
      std::copy(from, from + num_elements, to + num_elements * c);                                                \
    }                                                                                                             \
  }                                                                                                               \
  void scatter_##KIND##_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names, \
                                 std::string const& source_variable_name, int const root_circuit_index,           \
                                 int const num_elements)                                                          \
  {                                                                                                               \
    bool const named = !source_variable_name.empty();                                                             \
    auto const* from = std::addressof(states[root_circuit_index].to_##KIND##_variable(                            \
      named ? source_variable_name : variable_names[root_circuit_index]));                                        \
    for (int c = 0; c < static_cast<int>(states.size()); ++c) {                                                   \
      if (c == root_circuit_index && !named) continue;                                                            \
      std::copy(from + num_elements * c, from + num_elements * c + num_elements,                                  \
                std::addressof(states[c].to_##KIND##_variable(variable_names[c])));                               \
    }                                                                                                             \
  }
RBK_VARIABLE_TRANSFERS(real)
RBK_VARIABLE_TRANSFERS(complex)
RBK_VARIABLE_TRANSFERS(int)
#undef RBK_VARIABLE_TRANSFERS

}  // namespace bra
