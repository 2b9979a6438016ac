/* rbk_ket_mpi.hpp -- ket::mpi's single-process interface on a state held in
 * one B200's HBM.
 *
 * A ket::mpi program keeps its amplitudes in a local state
 * (ket::mpi::state<Complex, false>, ket/include/ket/mpi/state.hpp:1973-2100)
 * and a ket::mpi::qubit_permutation (ket/include/ket/mpi/qubit_permutation.hpp:40-302)
 * that maps each qubit to the bit of the local data holding it; every gate,
 * e.g.
 *   ket::mpi::gate::hadamard(mpi_policy, parallel_policy, local_state,
 *                            permutation, buffer, communicator, environment,
 *                            target, controls...)
 * (ket/include/ket/mpi/gate/hadamard.hpp:263-279), looks the qubits up in the
 * permutation and runs the ket gate on the local data.  With one process
 * every qubit is local, the permutation only changes when the program itself
 * changes it (ket::mpi::permutate), and SWAP exchanges data
 * (ket/include/ket/mpi/gate/swap.hpp:51-90).
 *
 * This header adds rbk::mpi::device_state<Complex>, the single-process
 * ket::mpi::state on the device, and overloads of the ket::mpi gate
 * functions and observables for (any MPI policy, ket::utility::policy::b200,
 * rbk::mpi::device_state).  A program moves to the GPU by passing make_b200()
 * and a device_state where it passed a ket parallel policy and a
 * ket::mpi::state; the permutation, buffer, communicator and environment
 * arguments stay.  The communicator must have one process (rbk::error
 * RBK_ERR_UNSUPPORTED otherwise).
 *
 * How the permutation is honoured: the device state's logical qubits are the
 * program's unpermuted qubits, and the engine's layout map (rbk.h, "layout
 * map") starts as the program's permutation, so the device memory in
 * physical order is exactly ket::mpi's local data.  Each call first compares
 * the permutation it is given with the one the state last followed; when the
 * program has changed it, the labels move with it (rbk_state_set_permutation,
 * no data movement), as ket::mpi's own local data stays put.
 * local_amplitudes() returns the local data in ket::mpi's order; and
 * device_data() moves the device memory into that order
 * (rbk_state_set_layout) and returns its address.
 *
 * Needs <ket/...> and <yampi/...> (the program's own yampi); C++14 or later.
 */
#ifndef RBK_KET_MPI_HPP
#define RBK_KET_MPI_HPP

#include <array>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <vector>

#include <ket/control.hpp>
#include <ket/mpi/qubit_permutation.hpp>
#include <ket/qubit.hpp>
#include <yampi/communicator.hpp>
#include <yampi/datatype_base.hpp>
#include <yampi/environment.hpp>

#include "rbk_ket.hpp"

namespace rbk {
namespace mpi {

namespace detail {
inline auto require_one_process(yampi::communicator const& communicator, yampi::environment const& environment)
  -> void
{
  if (communicator.size(environment) != 1)
    throw ::rbk::error(RBK_ERR_UNSUPPORTED, "rbk::mpi::device_state runs ket::mpi with one process only");
}

// The map of a ket::mpi::qubit_permutation: perm[q] = bit of the local data holding qubit q.
template <typename StateInteger, typename BitInteger, typename Allocator>
inline auto map_of(::ket::mpi::qubit_permutation<StateInteger, BitInteger, Allocator> const& permutation)
  -> std::vector<std::uint32_t>
{
  std::vector<std::uint32_t> map(permutation.size());
  for (std::size_t q = 0u; q < map.size(); ++q)
    map[q] = static_cast<std::uint32_t>(static_cast<BitInteger>(permutation[::ket::qubit<StateInteger, BitInteger>{q}].qubit()));
  return map;
}

// ket::mpi::permutate_bits (qubit_permutation.hpp:470-491): bit q of index
// goes to bit map[q].
inline auto permutate_bits(std::vector<std::uint32_t> const& map, std::uint64_t const index) -> std::uint64_t
{
  std::uint64_t result = 0u;
  for (std::size_t q = 0u; q < map.size(); ++q) result |= ((index >> q) & 1u) << map[q];
  return result;
}
}  // namespace detail

// 2^n amplitudes in one GPU's HBM behind ket::mpi's single-process interface.
// Move-only.
template <typename Complex>
class device_state {
 public:
  using value_type = Complex;
  using real_type = typename Complex::value_type;

  // ket::mpi::state<Complex, false>(num_local_qubits, initial_integer,
  // permutation, communicator, environment) (state.hpp:2031-2041): the state
  // |initial_integer>, with the local data in the permutation's order.
  template <typename BitInteger, typename StateInteger, typename PermutationAllocator>
  device_state(BitInteger const num_local_qubits, StateInteger const initial_integer,
               ::ket::mpi::qubit_permutation<StateInteger, BitInteger, PermutationAllocator> const& permutation,
               yampi::communicator const& communicator, yampi::environment const& environment, int const device = 0)
    : followed_{detail::map_of(permutation)},
      engine_{static_cast<unsigned>(num_local_qubits),
              detail::permutate_bits(detail::map_of(permutation), static_cast<std::uint64_t>(initial_integer)), device}
  {
    detail::require_one_process(communicator, environment);
    if (followed_.size() != static_cast<std::size_t>(num_local_qubits))
      throw ::rbk::error(RBK_ERR_INVALID, "rbk::mpi::device_state: the permutation does not have one entry per qubit");
    // The memory holds the local data under the identity map; declaring the
    // program's map makes the logical state |initial_integer>.
    ::rbk::check(rbk_state_set_permutation(engine_.handle(), followed_.data()));
  }

  auto num_local_qubits() const noexcept -> std::size_t { return engine_.num_qubits(); }
  auto num_data_blocks() const noexcept -> std::size_t { return 1u; }
  auto size() const noexcept -> std::uint64_t { return engine_.size(); }

  // The engine state in the program's unpermuted qubit order (rbk_ket.hpp's
  // ket::gate::ranges / ket::ranges overloads take it).
  auto engine() noexcept -> ::rbk::device_state<Complex>& { return engine_; }
  auto engine() const noexcept -> ::rbk::device_state<Complex> const& { return engine_; }
  // The permutation map the state follows now.
  auto followed_permutation() const -> std::vector<std::uint32_t> const& { return followed_; }

  // Brings the labels in line with the program's permutation (see the header
  // comment).  The gate and observable overloads call it.
  template <typename StateInteger, typename BitInteger, typename Allocator>
  auto follow(::ket::mpi::qubit_permutation<StateInteger, BitInteger, Allocator> const& permutation) -> void
  {
    auto const wanted = detail::map_of(permutation);
    if (wanted.size() != followed_.size())
      throw ::rbk::error(RBK_ERR_INVALID, "rbk::mpi::device_state: permutation size differs from the qubit count");
    if (wanted == followed_) return;
    // Engine: logical q on physical bit M[q].  Program: qubit q on local-data
    // bit P[q] before, P'[q] now, with the local data unchanged.  The qubit
    // that P' puts on bit P'[q] was the one P put there, inverse(P)[P'[q]],
    // whose physical bit is M[inverse(P)[P'[q]]].
    std::vector<std::uint32_t> inverse_followed(followed_.size());
    for (std::size_t q = 0u; q < followed_.size(); ++q) inverse_followed[followed_[q]] = static_cast<std::uint32_t>(q);
    auto const current = engine_.permutation();
    std::vector<std::uint32_t> next(current.size());
    for (std::size_t q = 0u; q < next.size(); ++q) next[q] = current[inverse_followed[wanted[q]]];
    ::rbk::check(rbk_state_set_permutation(engine_.handle(), next.data()));
    followed_ = wanted;
  }

  // The local data of ket::mpi::state: amplitude i of the state at index
  // permutate_bits(permutation, i).
  auto local_amplitudes() const -> std::vector<Complex>
  {
    auto const logical = engine_.amplitudes();
    std::vector<Complex> local(logical.size());
    for (std::uint64_t i = 0u; i < logical.size(); ++i) local[detail::permutate_bits(followed_, i)] = logical[i];
    return local;
  }

  // Device address of the local data in ket::mpi's order: the memory is moved
  // into the followed permutation's layout first.  Valid until the next gate.
  auto device_data() -> void*
  {
    ::rbk::check(rbk_state_set_layout(engine_.handle(), followed_.data()));
    void* p = nullptr;
    ::rbk::check(rbk_state_device_pointer(engine_.handle(), &p));
    ::rbk::check(rbk_state_synchronize(engine_.handle()));
    return p;
  }

 private:
  std::vector<std::uint32_t> followed_;
  ::rbk::device_state<Complex> engine_;
};

}  // namespace mpi
}  // namespace rbk

// Gate overloads: (MPI policy, b200, rbk::mpi::device_state&, permutation&,
// buffer&, [datatype,] communicator, environment, the arguments of the ket
// gate), as ket::mpi::gate's public forms take them.  The buffer and datatype
// are not needed on the device.
#define RBK_KET_MPI_GATE(NAME)                                                                                        \
  template <typename MpiPolicy, typename Complex, typename StateInteger, typename BitInteger, typename Allocator,     \
            typename BufferAllocator, typename... Args>                                                               \
  inline auto NAME(MpiPolicy const&, ::ket::utility::policy::b200 const policy,                                      \
                   ::rbk::mpi::device_state<Complex>& local_state,                                                    \
                   ::ket::mpi::qubit_permutation<StateInteger, BitInteger, Allocator>& permutation,                   \
                   std::vector<Complex, BufferAllocator>&, yampi::communicator const& communicator,                   \
                   yampi::environment const& environment, Args const... args)                                         \
    ->::rbk::mpi::device_state<Complex>&                                                                              \
  {                                                                                                                   \
    ::rbk::mpi::detail::require_one_process(communicator, environment);                                               \
    local_state.follow(permutation);                                                                                  \
    ::ket::gate::ranges::NAME(policy, local_state.engine(), args...);                                                 \
    return local_state;                                                                                               \
  }                                                                                                                   \
  template <typename MpiPolicy, typename Complex, typename StateInteger, typename BitInteger, typename Allocator,     \
            typename BufferAllocator, typename DerivedDatatype, typename... Args>                                     \
  inline auto NAME(MpiPolicy const& mpi_policy, ::ket::utility::policy::b200 const policy,                           \
                   ::rbk::mpi::device_state<Complex>& local_state,                                                    \
                   ::ket::mpi::qubit_permutation<StateInteger, BitInteger, Allocator>& permutation,                   \
                   std::vector<Complex, BufferAllocator>& buffer, yampi::datatype_base<DerivedDatatype> const&,       \
                   yampi::communicator const& communicator, yampi::environment const& environment,                    \
                   Args const... args)                                                                                \
    ->::rbk::mpi::device_state<Complex>&                                                                              \
  {                                                                                                                   \
    return NAME(mpi_policy, policy, local_state, permutation, buffer, communicator, environment, args...);            \
  }

namespace ket {
namespace mpi {
namespace gate {
// ket/include/ket/mpi/gate/hadamard.hpp:263-279
RBK_KET_MPI_GATE(hadamard)
RBK_KET_MPI_GATE(adj_hadamard)
// pauli_x.hpp, not_.hpp, controlled_not.hpp, toffoli.hpp
RBK_KET_MPI_GATE(pauli_x)
RBK_KET_MPI_GATE(adj_pauli_x)
RBK_KET_MPI_GATE(not_)
RBK_KET_MPI_GATE(adj_not_)
RBK_KET_MPI_GATE(controlled_not)
RBK_KET_MPI_GATE(adj_controlled_not)
RBK_KET_MPI_GATE(toffoli)
RBK_KET_MPI_GATE(adj_toffoli)
// pauli_y.hpp; pauli_z.hpp (detail/pauli_z_*.hpp)
RBK_KET_MPI_GATE(pauli_y)
RBK_KET_MPI_GATE(adj_pauli_y)
RBK_KET_MPI_GATE(pauli_z)
RBK_KET_MPI_GATE(adj_pauli_z)
// phase_shift.hpp (detail/phase_shift_*.hpp): U1 / coefficient, U2, U3
RBK_KET_MPI_GATE(phase_shift_coeff)
RBK_KET_MPI_GATE(adj_phase_shift_coeff)
RBK_KET_MPI_GATE(phase_shift)
RBK_KET_MPI_GATE(adj_phase_shift)
RBK_KET_MPI_GATE(phase_shift2)
RBK_KET_MPI_GATE(adj_phase_shift2)
RBK_KET_MPI_GATE(phase_shift3)
RBK_KET_MPI_GATE(adj_phase_shift3)
// controlled_phase_shift.hpp
RBK_KET_MPI_GATE(controlled_phase_shift_coeff)
RBK_KET_MPI_GATE(adj_controlled_phase_shift_coeff)
RBK_KET_MPI_GATE(controlled_phase_shift)
RBK_KET_MPI_GATE(adj_controlled_phase_shift)
// exponential_pauli_{x,y,z}.hpp, exponential_swap.hpp
RBK_KET_MPI_GATE(exponential_pauli_x)
RBK_KET_MPI_GATE(adj_exponential_pauli_x)
RBK_KET_MPI_GATE(exponential_pauli_y)
RBK_KET_MPI_GATE(adj_exponential_pauli_y)
RBK_KET_MPI_GATE(exponential_pauli_z)
RBK_KET_MPI_GATE(adj_exponential_pauli_z)
RBK_KET_MPI_GATE(exponential_swap)
RBK_KET_MPI_GATE(adj_exponential_swap)
// swap.hpp:51-90 (with one process: the data of the two qubits is exchanged
// and the permutation is unchanged; here the labels move, which is the same
// state)
RBK_KET_MPI_GATE(swap)
RBK_KET_MPI_GATE(adj_swap)
// x/y_rotation_half_pi.hpp, sqrt_pauli_{x,y,z}.hpp, clear.hpp, set.hpp
RBK_KET_MPI_GATE(x_rotation_half_pi)
RBK_KET_MPI_GATE(adj_x_rotation_half_pi)
RBK_KET_MPI_GATE(y_rotation_half_pi)
RBK_KET_MPI_GATE(adj_y_rotation_half_pi)
RBK_KET_MPI_GATE(sqrt_pauli_x)
RBK_KET_MPI_GATE(adj_sqrt_pauli_x)
RBK_KET_MPI_GATE(sqrt_pauli_y)
RBK_KET_MPI_GATE(adj_sqrt_pauli_y)
RBK_KET_MPI_GATE(sqrt_pauli_z)
RBK_KET_MPI_GATE(adj_sqrt_pauli_z)
RBK_KET_MPI_GATE(clear)
RBK_KET_MPI_GATE(set)
}  // namespace gate

// ---- observables -------------------------------------------------------------
// all_spin_expectation_values.hpp:29-60: <S_x>, <S_y>, <S_z> of qubits 0..num_qubits-1.
template <typename SpinsAllocator, typename MpiPolicy, typename Complex, typename StateInteger, typename BitInteger,
          typename Allocator, typename BufferAllocator>
inline auto all_spin_expectation_values(MpiPolicy const&, ::ket::utility::policy::b200 const policy,
                                        ::rbk::mpi::device_state<Complex>& local_state,
                                        ::ket::mpi::qubit_permutation<StateInteger, BitInteger, Allocator>& permutation,
                                        BitInteger const num_qubits, std::vector<Complex, BufferAllocator>&,
                                        yampi::communicator const& communicator, yampi::environment const& environment)
  -> std::vector<std::array<typename Complex::value_type, 3u>, SpinsAllocator>
{
  ::rbk::mpi::detail::require_one_process(communicator, environment);
  local_state.follow(permutation);
  auto const all = ::ket::ranges::all_spin_expectation_values< ::ket::qubit<StateInteger, BitInteger> >(
    policy, local_state.engine());
  return std::vector<std::array<typename Complex::value_type, 3u>, SpinsAllocator>(
    all.begin(), all.begin() + static_cast<std::ptrdiff_t>(num_qubits));
}

// spin_expectation_value.hpp: <S_x>, <S_y>, <S_z> of one qubit.
template <typename MpiPolicy, typename Complex, typename StateInteger, typename BitInteger, typename Allocator,
          typename BufferAllocator>
inline auto spin_expectation_value(MpiPolicy const&, ::ket::utility::policy::b200 const policy,
                                   ::rbk::mpi::device_state<Complex>& local_state,
                                   ::ket::mpi::qubit_permutation<StateInteger, BitInteger, Allocator>& permutation,
                                   std::vector<Complex, BufferAllocator>&, yampi::communicator const& communicator,
                                   yampi::environment const& environment, ::ket::qubit<StateInteger, BitInteger> const qubit)
  -> std::array<typename Complex::value_type, 3u>
{
  ::rbk::mpi::detail::require_one_process(communicator, environment);
  local_state.follow(permutation);
  return ::ket::ranges::spin_expectation_value(policy, local_state.engine(), qubit);
}

// inner_product.hpp:130-146 and fidelity.hpp: over the local data of two
// states, which ket::mpi lays out by one permutation; both states must follow
// the same one.
template <typename MpiPolicy, typename Complex>
inline auto inner_product(MpiPolicy const&, ::ket::utility::policy::b200 const policy,
                          ::rbk::mpi::device_state<Complex> const& local_state1,
                          ::rbk::mpi::device_state<Complex> const& local_state2, yampi::communicator const& communicator,
                          yampi::environment const& environment) -> Complex
{
  ::rbk::mpi::detail::require_one_process(communicator, environment);
  if (local_state1.followed_permutation() != local_state2.followed_permutation())
    throw ::rbk::error(RBK_ERR_INVALID, "ket::mpi::inner_product: the states follow different permutations");
  return ::ket::ranges::inner_product(policy, local_state1.engine(), local_state2.engine());
}

template <typename MpiPolicy, typename Complex>
inline auto fidelity(MpiPolicy const&, ::ket::utility::policy::b200 const policy,
                     ::rbk::mpi::device_state<Complex> const& local_state1,
                     ::rbk::mpi::device_state<Complex> const& local_state2, yampi::communicator const& communicator,
                     yampi::environment const& environment) -> typename Complex::value_type
{
  ::rbk::mpi::detail::require_one_process(communicator, environment);
  if (local_state1.followed_permutation() != local_state2.followed_permutation())
    throw ::rbk::error(RBK_ERR_INVALID, "ket::mpi::fidelity: the states follow different permutations");
  return ::ket::ranges::fidelity(policy, local_state1.engine(), local_state2.engine());
}
}  // namespace mpi
}  // namespace ket

#undef RBK_KET_MPI_GATE

#endif  // RBK_KET_MPI_HPP
