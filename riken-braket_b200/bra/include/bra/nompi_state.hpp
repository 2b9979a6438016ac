// bra's single-process state on one B200: the class bra::nompi_state that
// bra's main (bra/src/bra.cpp) constructs, with the same constructor and the
// same free functions for the multi-circuit instructions, backed by the rbk
// engine (include/rbk.h) instead of a host vector and ket's CPU loops.
//
// The reference's class (bra/include/bra/nompi_state.hpp, bra/src/nompi_state.cpp)
// implements bra::state's do_* backend (bra/include/bra/state.hpp:1022-1318)
// on data_, a std::vector of amplitudes.  This header replaces it at build
// time: it comes first on the include path, and bra/src/nompi_state.cpp is
// not compiled, so bra's interpreter, its gate objects and its main run
// unchanged on the device (riken-braket_b200/bra/Makefile).  The amplitudes
// live in HBM; gates are queued and executed by the fused passes; BEGIN/END
// FUSION map to the engine's fusion blocks; measurements and events draw from
// bra::state's own random number generator exactly as ket's CPU code does.
//
// Differences from the reference: the state cannot be copied (only moved),
// and GENERATE EVENTS leaves the state intact (the reference's
// ket::generate_events overwrites it with prefix sums).
#ifndef RBK_BRA_NOMPI_STATE_HPP
#define RBK_BRA_NOMPI_STATE_HPP

#ifdef BRA_NO_MPI
#include <string>
#include <type_traits>
#include <vector>

#include <bra/state.hpp>
#include <bra/types.hpp>

#include "rbk.h"

namespace bra {

class nompi_state final : public ::bra::state
{
  static_assert(std::is_same< ::bra::real_type, double>::value, "the B200 backend is built for complex<double> states");

  friend void inner_product(nompi_state& state1, nompi_state& state2);
  friend void inner_product_all(std::vector<nompi_state>& states);
  friend void inner_product_op(nompi_state& state1, nompi_state& state2, std::string const& operator_literal_or_variable_name,
                               std::vector< ::bra::qubit_type > const& operated_qubits);
  friend void inner_product_all_op(std::vector<nompi_state>& states, std::string const& operator_literal_or_variable_name,
                                   std::vector< ::bra::qubit_type > const& operated_qubits);
  friend void fidelity(nompi_state& state1, nompi_state& state2);
  friend void fidelity_all(std::vector<nompi_state>& states);
  friend void fidelity_op(nompi_state& state1, nompi_state& state2, std::string const& operator_literal_or_variable_name,
                          std::vector< ::bra::qubit_type > const& operated_qubits);
  friend void fidelity_all_op(std::vector<nompi_state>& states, std::string const& operator_literal_or_variable_name,
                              std::vector< ::bra::qubit_type > const& operated_qubits);
  friend void send_real_variable(nompi_state const& source_state, std::string const& source_variable_name,
                                 nompi_state& destination_state, std::string const& destination_variable_name,
                                 int const num_elements);
  friend void send_complex_variable(nompi_state const& source_state, std::string const& source_variable_name,
                                    nompi_state& destination_state, std::string const& destination_variable_name,
                                    int const num_elements);
  friend void send_int_variable(nompi_state const& source_state, std::string const& source_variable_name,
                                nompi_state& destination_state, std::string const& destination_variable_name,
                                int const num_elements);
  friend void broadcast_real_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names,
                                      int const root_circuit_index, int const num_elements);
  friend void broadcast_complex_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names,
                                         int const root_circuit_index, int const num_elements);
  friend void broadcast_int_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names,
                                     int const root_circuit_index, int const num_elements);
  friend void gather_real_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names,
                                   std::string const& destination_variable_name, int const root_circuit_index,
                                   int const num_elements);
  friend void gather_complex_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names,
                                      std::string const& destination_variable_name, int const root_circuit_index,
                                      int const num_elements);
  friend void gather_int_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names,
                                  std::string const& destination_variable_name, int const root_circuit_index,
                                  int const num_elements);
  friend void scatter_real_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names,
                                    std::string const& source_variable_name, int const root_circuit_index,
                                    int const num_elements);
  friend void scatter_complex_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names,
                                       std::string const& source_variable_name, int const root_circuit_index,
                                       int const num_elements);
  friend void scatter_int_variable(std::vector<nompi_state>& states, std::vector<std::string> const& variable_names,
                                   std::string const& source_variable_name, int const root_circuit_index,
                                   int const num_elements);

 public:
  // The reference's constructor.  num_threads is accepted and unused (the
  // engine's parallelism is the GPU's).  The device is RBK_DEVICE (default 0).
  nompi_state(::bra::state::state_integer_type const initial_integer, unsigned int const total_num_qubits,
              unsigned int const num_threads, ::bra::state::seed_type const seed, bool const is_depolarizing_channel,
              ::bra::real_type const depolarizing_px, ::bra::real_type const depolarizing_py,
              ::bra::real_type const depolarizing_pz, bool const uses_depolarizing_seed,
              ::bra::state::seed_type const depolarizing_seed, int const circuit_index);
  ~nompi_state();
  nompi_state(nompi_state const&) = delete;
  nompi_state& operator=(nompi_state const&) = delete;
  nompi_state(nompi_state&& other) noexcept;
  nompi_state& operator=(nompi_state&& other) noexcept;

  // The engine's state (for callers that read it through include/rbk.h).
  rbk_state* handle() const noexcept { return handle_; }

 private:
  rbk_state* handle_ = nullptr;
  mutable bool is_waiting_ = false;

  auto do_is_waiting() const -> bool override;
  auto do_cancel_waiting() -> void override;
  auto generate_probability() -> real_type override;
  auto do_send_real_variable(int const circuit_index, std::string const& variable_name, int const num_elements) const -> void override;
  auto do_send_complex_variable(int const circuit_index, std::string const& variable_name, int const num_elements) const -> void override;
  auto do_send_int_variable(int const circuit_index, std::string const& variable_name, int const num_elements) const -> void override;
  auto do_receive_real_variable(int const circuit_index, std::string const& variable_name, int const num_elements) -> void override;
  auto do_receive_complex_variable(int const circuit_index, std::string const& variable_name, int const num_elements) -> void override;
  auto do_receive_int_variable(int const circuit_index, std::string const& variable_name, int const num_elements) -> void override;
  auto do_broadcast_real_variable(int const circuit_index, std::string const& variable_name, int const num_elements) -> void override;
  auto do_broadcast_complex_variable(int const circuit_index, std::string const& variable_name, int const num_elements) -> void override;
  auto do_broadcast_int_variable(int const circuit_index, std::string const& variable_name, int const num_elements) -> void override;
  auto do_gather_real_variable(int const circuit_index, std::string const& variable_name, int const num_elements,
                               std::string const& destination_variable_name) -> void override;
  auto do_gather_complex_variable(int const circuit_index, std::string const& variable_name, int const num_elements,
                                  std::string const& destination_variable_name) -> void override;
  auto do_gather_int_variable(int const circuit_index, std::string const& variable_name, int const num_elements,
                              std::string const& destination_variable_name) -> void override;
  auto do_scatter_real_variable(int const circuit_index, std::string const& variable_name, int const num_elements,
                                std::string const& source_variable_name) -> void override;
  auto do_scatter_complex_variable(int const circuit_index, std::string const& variable_name, int const num_elements,
                                   std::string const& source_variable_name) -> void override;
  auto do_scatter_int_variable(int const circuit_index, std::string const& variable_name, int const num_elements,
                               std::string const& source_variable_name) -> void override;

  void do_i_gate(qubit_type const qubit) override;
  void do_ic_gate(control_qubit_type const control_qubit) override;
  void do_ii_gate(qubit_type const qubit1, qubit_type const qubit2) override;
  void do_in_gate(std::vector<qubit_type> const& qubits) override;
  void do_hadamard(qubit_type const qubit) override;
  void do_not_(qubit_type const qubit) override;
  void do_pauli_x(qubit_type const qubit) override;
  void do_pauli_xx(qubit_type const qubit1, qubit_type const qubit2) override;
  void do_pauli_xn(std::vector<qubit_type> const& qubits) override;
  void do_pauli_y(qubit_type const qubit) override;
  void do_pauli_yy(qubit_type const qubit1, qubit_type const qubit2) override;
  void do_pauli_yn(std::vector<qubit_type> const& qubits) override;
  void do_pauli_z(control_qubit_type const control_qubit) override;
  void do_pauli_zz(qubit_type const qubit1, qubit_type const qubit2) override;
  void do_pauli_zn(std::vector<qubit_type> const& qubits) override;
  void do_swap(qubit_type const qubit1, qubit_type const qubit2) override;
  void do_sqrt_pauli_x(qubit_type const qubit) override;
  void do_adj_sqrt_pauli_x(qubit_type const qubit) override;
  void do_sqrt_pauli_y(qubit_type const qubit) override;
  void do_adj_sqrt_pauli_y(qubit_type const qubit) override;
  void do_sqrt_pauli_z(control_qubit_type const control_qubit) override;
  void do_adj_sqrt_pauli_z(control_qubit_type const control_qubit) override;
  void do_sqrt_pauli_zz(qubit_type const qubit1, qubit_type const qubit2) override;
  void do_adj_sqrt_pauli_zz(qubit_type const qubit1, qubit_type const qubit2) override;
  void do_sqrt_pauli_zn(std::vector<qubit_type> const& qubits) override;
  void do_adj_sqrt_pauli_zn(std::vector<qubit_type> const& qubits) override;
  void do_u1(real_type const phase, control_qubit_type const control_qubit) override;
  void do_adj_u1(real_type const phase, control_qubit_type const control_qubit) override;
  void do_u2(real_type const phase1, real_type const phase2, qubit_type const qubit) override;
  void do_adj_u2(real_type const phase1, real_type const phase2, qubit_type const qubit) override;
  void do_u3(real_type const phase1, real_type const phase2, real_type const phase3, qubit_type const qubit) override;
  void do_adj_u3(real_type const phase1, real_type const phase2, real_type const phase3, qubit_type const qubit) override;
  void do_phase_shift(complex_type const& phase_coefficient, control_qubit_type const control_qubit) override;
  void do_adj_phase_shift(complex_type const& phase_coefficient, control_qubit_type const control_qubit) override;
  void do_x_rotation_half_pi(qubit_type const qubit) override;
  void do_adj_x_rotation_half_pi(qubit_type const qubit) override;
  void do_y_rotation_half_pi(qubit_type const qubit) override;
  void do_adj_y_rotation_half_pi(qubit_type const qubit) override;
  void do_exponential_pauli_x(real_type const phase, qubit_type const qubit) override;
  void do_adj_exponential_pauli_x(real_type const phase, qubit_type const qubit) override;
  void do_exponential_pauli_xx(real_type const phase, qubit_type const qubit1, qubit_type const qubit2) override;
  void do_adj_exponential_pauli_xx(real_type const phase, qubit_type const qubit1, qubit_type const qubit2) override;
  void do_exponential_pauli_xn(real_type const phase, std::vector<qubit_type> const& qubits) override;
  void do_adj_exponential_pauli_xn(real_type const phase, std::vector<qubit_type> const& qubits) override;
  void do_exponential_pauli_y(real_type const phase, qubit_type const qubit) override;
  void do_adj_exponential_pauli_y(real_type const phase, qubit_type const qubit) override;
  void do_exponential_pauli_yy(real_type const phase, qubit_type const qubit1, qubit_type const qubit2) override;
  void do_adj_exponential_pauli_yy(real_type const phase, qubit_type const qubit1, qubit_type const qubit2) override;
  void do_exponential_pauli_yn(real_type const phase, std::vector<qubit_type> const& qubits) override;
  void do_adj_exponential_pauli_yn(real_type const phase, std::vector<qubit_type> const& qubits) override;
  void do_exponential_pauli_z(real_type const phase, qubit_type const qubit) override;
  void do_adj_exponential_pauli_z(real_type const phase, qubit_type const qubit) override;
  void do_exponential_pauli_zz(real_type const phase, qubit_type const qubit1, qubit_type const qubit2) override;
  void do_adj_exponential_pauli_zz(real_type const phase, qubit_type const qubit1, qubit_type const qubit2) override;
  void do_exponential_pauli_zn(real_type const phase, std::vector<qubit_type> const& qubits) override;
  void do_adj_exponential_pauli_zn(real_type const phase, std::vector<qubit_type> const& qubits) override;
  void do_exponential_swap(real_type const phase, qubit_type const qubit1, qubit_type const qubit2) override;
  void do_adj_exponential_swap(real_type const phase, qubit_type const qubit1, qubit_type const qubit2) override;
  void do_toffoli(qubit_type const target_qubit, control_qubit_type const control_qubit1,
                  control_qubit_type const control_qubit2) override;
  ket::gate::outcome do_projective_measurement(qubit_type const qubit) override;
  void do_expectation_values() override;
  void do_amplitudes(std::vector< ::bra::state_integer_type > const& amplitude_indices) override;
  void do_measure() override;
  void do_generate_events(int const num_events, int const seed) override;
  void do_expectation_value(std::string const& operator_literal_or_variable_name,
                            std::vector<qubit_type> const& operated_qubits) override;
  void do_inner_product(std::string const& remote_circuit_index_or_all) override;
  void do_inner_product(std::string const& remote_circuit_index_or_all, std::string const& operator_literal_or_variable_name,
                        std::vector<qubit_type> const& operated_qubits) override;
  void do_fidelity(std::string const& remote_circuit_index_or_all) override;
  void do_fidelity(std::string const& remote_circuit_index_or_all, std::string const& operator_literal_or_variable_name,
                   std::vector<qubit_type> const& operated_qubits) override;
  void do_shor_box(state_integer_type const divisor, state_integer_type const base,
                   std::vector<qubit_type> const& exponent_qubits,
                   std::vector<qubit_type> const& modular_exponentiation_qubits) override;
  void do_begin_fusion() override;
  void do_end_fusion() override;
  void do_clear(qubit_type const qubit) override;
  void do_set(qubit_type const qubit) override;
  void do_controlled_i_gate(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_controlled_ic_gate(control_qubit_type const control_qubit1, control_qubit_type const control_qubit2) override;
  void do_multi_controlled_in_gate(std::vector<qubit_type> const& target_qubits,
                                   std::vector<control_qubit_type> const& control_qubits) override;
  void do_multi_controlled_ic_gate(std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_hadamard(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_multi_controlled_hadamard(qubit_type const target_qubit, std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_not(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_multi_controlled_not(qubit_type const target_qubit, std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_pauli_x(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_multi_controlled_pauli_xn(std::vector<qubit_type> const& target_qubits,
                                    std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_pauli_y(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_multi_controlled_pauli_yn(std::vector<qubit_type> const& target_qubits,
                                    std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_pauli_z(control_qubit_type const control_qubit1, control_qubit_type const control_qubit2) override;
  void do_multi_controlled_pauli_z(std::vector<control_qubit_type> const& control_qubits) override;
  void do_multi_controlled_pauli_zn(std::vector<qubit_type> const& target_qubits,
                                    std::vector<control_qubit_type> const& control_qubits) override;
  void do_multi_controlled_swap(qubit_type const target_qubit1, qubit_type const target_qubit2,
                                std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_sqrt_pauli_x(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_adj_controlled_sqrt_pauli_x(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_multi_controlled_sqrt_pauli_x(qubit_type const target_qubit, std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_sqrt_pauli_x(qubit_type const target_qubit,
                                            std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_sqrt_pauli_y(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_adj_controlled_sqrt_pauli_y(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_multi_controlled_sqrt_pauli_y(qubit_type const target_qubit, std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_sqrt_pauli_y(qubit_type const target_qubit,
                                            std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_sqrt_pauli_z(control_qubit_type const control_qubit1, control_qubit_type const control_qubit2) override;
  void do_adj_controlled_sqrt_pauli_z(control_qubit_type const control_qubit1, control_qubit_type const control_qubit2) override;
  void do_multi_controlled_sqrt_pauli_z(std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_sqrt_pauli_z(std::vector<control_qubit_type> const& control_qubits) override;
  void do_multi_controlled_sqrt_pauli_zn(std::vector<qubit_type> const& target_qubits,
                                         std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_sqrt_pauli_zn(std::vector<qubit_type> const& target_qubits,
                                             std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_phase_shift(complex_type const& phase_coefficient, control_qubit_type const control_qubit1,
                                 control_qubit_type const control_qubit2) override;
  void do_adj_controlled_phase_shift(complex_type const& phase_coefficient, control_qubit_type const control_qubit1,
                                     control_qubit_type const control_qubit2) override;
  void do_multi_controlled_phase_shift(complex_type const& phase_coefficient,
                                       std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_phase_shift(complex_type const& phase_coefficient,
                                           std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_u1(real_type const phase, control_qubit_type const control_qubit1,
                        control_qubit_type const control_qubit2) override;
  void do_adj_controlled_u1(real_type const phase, control_qubit_type const control_qubit1,
                            control_qubit_type const control_qubit2) override;
  void do_multi_controlled_u1(real_type const phase, std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_u1(real_type const phase, std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_u2(real_type const phase1, real_type const phase2, qubit_type const target_qubit,
                        control_qubit_type const control_qubit) override;
  void do_adj_controlled_u2(real_type const phase1, real_type const phase2, qubit_type const target_qubit,
                            control_qubit_type const control_qubit) override;
  void do_multi_controlled_u2(real_type const phase1, real_type const phase2, qubit_type const target_qubit,
                              std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_u2(real_type const phase1, real_type const phase2, qubit_type const target_qubit,
                                  std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_u3(real_type const phase1, real_type const phase2, real_type const phase3, qubit_type const target_qubit,
                        control_qubit_type const control_qubit) override;
  void do_adj_controlled_u3(real_type const phase1, real_type const phase2, real_type const phase3,
                            qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_multi_controlled_u3(real_type const phase1, real_type const phase2, real_type const phase3,
                              qubit_type const target_qubit, std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_u3(real_type const phase1, real_type const phase2, real_type const phase3,
                                  qubit_type const target_qubit, std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_x_rotation_half_pi(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_adj_controlled_x_rotation_half_pi(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_multi_controlled_x_rotation_half_pi(qubit_type const target_qubit,
                                              std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_x_rotation_half_pi(qubit_type const target_qubit,
                                                  std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_y_rotation_half_pi(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_adj_controlled_y_rotation_half_pi(qubit_type const target_qubit, control_qubit_type const control_qubit) override;
  void do_multi_controlled_y_rotation_half_pi(qubit_type const target_qubit,
                                              std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_y_rotation_half_pi(qubit_type const target_qubit,
                                                  std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_exponential_pauli_x(real_type const phase, qubit_type const target_qubit,
                                         control_qubit_type const control_qubit) override;
  void do_adj_controlled_exponential_pauli_x(real_type const phase, qubit_type const target_qubit,
                                             control_qubit_type const control_qubit) override;
  void do_multi_controlled_exponential_pauli_xn(real_type const phase, std::vector<qubit_type> const& target_qubits,
                                                std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_exponential_pauli_xn(real_type const phase, std::vector<qubit_type> const& target_qubits,
                                                    std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_exponential_pauli_y(real_type const phase, qubit_type const target_qubit,
                                         control_qubit_type const control_qubit) override;
  void do_adj_controlled_exponential_pauli_y(real_type const phase, qubit_type const target_qubit,
                                             control_qubit_type const control_qubit) override;
  void do_multi_controlled_exponential_pauli_yn(real_type const phase, std::vector<qubit_type> const& target_qubits,
                                                std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_exponential_pauli_yn(real_type const phase, std::vector<qubit_type> const& target_qubits,
                                                    std::vector<control_qubit_type> const& control_qubits) override;
  void do_controlled_exponential_pauli_z(real_type const phase, qubit_type const target_qubit,
                                         control_qubit_type const control_qubit) override;
  void do_adj_controlled_exponential_pauli_z(real_type const phase, qubit_type const target_qubit,
                                             control_qubit_type const control_qubit) override;
  void do_multi_controlled_exponential_pauli_z(real_type const phase, qubit_type const target_qubit,
                                               std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_exponential_pauli_z(real_type const phase, qubit_type const target_qubit,
                                                   std::vector<control_qubit_type> const& control_qubits) override;
  void do_multi_controlled_exponential_pauli_zn(real_type const phase, std::vector<qubit_type> const& target_qubits,
                                                std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_exponential_pauli_zn(real_type const phase, std::vector<qubit_type> const& target_qubits,
                                                    std::vector<control_qubit_type> const& control_qubits) override;
  void do_multi_controlled_exponential_swap(real_type const phase, qubit_type const target_qubit1,
                                            qubit_type const target_qubit2,
                                            std::vector<control_qubit_type> const& control_qubits) override;
  void do_adj_multi_controlled_exponential_swap(real_type const phase, qubit_type const target_qubit1,
                                                qubit_type const target_qubit2,
                                                std::vector<control_qubit_type> const& control_qubits) override;
};

void inner_product(nompi_state& state1, nompi_state& state2);
void inner_product_all(std::vector< ::bra::nompi_state >& states);
void inner_product_op(nompi_state& state1, nompi_state& state2, std::string const& operator_literal_or_variable_name,
                      std::vector< ::bra::qubit_type > const& operated_qubits);
void inner_product_all_op(std::vector< ::bra::nompi_state >& states, std::string const& operator_literal_or_variable_name,
                          std::vector< ::bra::qubit_type > const& operated_qubits);
void fidelity(nompi_state& state1, nompi_state& state2);
void fidelity_all(std::vector< ::bra::nompi_state >& states);
void fidelity_op(nompi_state& state1, nompi_state& state2, std::string const& operator_literal_or_variable_name,
                 std::vector< ::bra::qubit_type > const& operated_qubits);
void fidelity_all_op(std::vector< ::bra::nompi_state >& states, std::string const& operator_literal_or_variable_name,
                     std::vector< ::bra::qubit_type > const& operated_qubits);
void send_real_variable(nompi_state const& source_state, std::string const& source_variable_name,
                        nompi_state& destination_state, std::string const& destination_variable_name, int const num_elements);
void send_complex_variable(nompi_state const& source_state, std::string const& source_variable_name,
                           nompi_state& destination_state, std::string const& destination_variable_name,
                           int const num_elements);
void send_int_variable(nompi_state const& source_state, std::string const& source_variable_name,
                       nompi_state& destination_state, std::string const& destination_variable_name, int const num_elements);
void broadcast_real_variable(std::vector< ::bra::nompi_state >& states, std::vector<std::string> const& variable_names,
                             int const root_circuit_index, int const num_elements);
void broadcast_complex_variable(std::vector< ::bra::nompi_state >& states, std::vector<std::string> const& variable_names,
                                int const root_circuit_index, int const num_elements);
void broadcast_int_variable(std::vector< ::bra::nompi_state >& states, std::vector<std::string> const& variable_names,
                            int const root_circuit_index, int const num_elements);
void gather_real_variable(std::vector< ::bra::nompi_state >& states, std::vector<std::string> const& variable_names,
                          std::string const& destination_variable_name, int const root_circuit_index, int const num_elements);
void gather_complex_variable(std::vector< ::bra::nompi_state >& states, std::vector<std::string> const& variable_names,
                             std::string const& destination_variable_name, int const root_circuit_index, int const num_elements);
void gather_int_variable(std::vector< ::bra::nompi_state >& states, std::vector<std::string> const& variable_names,
                         std::string const& destination_variable_name, int const root_circuit_index, int const num_elements);
void scatter_real_variable(std::vector< ::bra::nompi_state >& states, std::vector<std::string> const& variable_names,
                           std::string const& source_variable_name, int const root_circuit_index, int const num_elements);
void scatter_complex_variable(std::vector< ::bra::nompi_state >& states, std::vector<std::string> const& variable_names,
                              std::string const& source_variable_name, int const root_circuit_index, int const num_elements);
void scatter_int_variable(std::vector< ::bra::nompi_state >& states, std::vector<std::string> const& variable_names,
                          std::string const& source_variable_name, int const root_circuit_index, int const num_elements);

}  // namespace bra

#endif  // BRA_NO_MPI
#endif  // RBK_BRA_NOMPI_STATE_HPP
