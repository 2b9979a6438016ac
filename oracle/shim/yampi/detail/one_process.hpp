// Project-written single-process stand-in for yampi, the MPI wrapper that
// RIKEN-braket's ket::mpi headers call (an un-vendored submodule of the
// reference; absent here).  TEST INFRASTRUCTURE ONLY: it lets ket's own
// ket::mpi code (state, qubit_permutation, gates, observables) compile and run
// as one process, the "single-process" configuration of ket::mpi, so that a
// ket::mpi program can be run on ket's CPU code and on the device adapter of
// include/rbk_ket_mpi.hpp and compared.
//
// Every communicator has one rank (0).  Collectives therefore reduce to local
// copies: in-place reductions and broadcasts leave the buffer as it is,
// out-of-place ones copy the send buffer to the receive side, and a
// send/receive with oneself copies.  Operations that only a job of several
// processes reaches (point-to-point messages to another rank, the data
// exchanges of global qubits) throw std::logic_error.
//
// The names and call forms are those used by ket/include/ket/mpi/** (for
// example ket/include/ket/mpi/utility/simple_mpi.hpp, inner_product.hpp,
// all_spin_expectation_values.hpp, utility/logger.hpp).
#ifndef RBK_SHIM_YAMPI_ONE_PROCESS_HPP
#define RBK_SHIM_YAMPI_ONE_PROCESS_HPP

#include <algorithm>
#include <chrono>
#include <cstddef>
#include <iterator>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace yampi {

enum class thread_support { single, funneled, serialized, multiple };

class environment {
  ::yampi::thread_support support_ = ::yampi::thread_support::single;

 public:
  environment() = default;
  explicit environment(::yampi::thread_support s) : support_{s} {}
  environment(int&, char**&, ::yampi::thread_support s) : support_{s} {}
  environment(environment const&) = delete;
  environment& operator=(environment const&) = delete;
  auto thread_support() const -> ::yampi::thread_support { return support_; }
};

class rank {
  int value_ = 0;

 public:
  constexpr rank() noexcept = default;
  constexpr explicit rank(int v) noexcept : value_{v} {}
  constexpr auto mpi_rank() const noexcept -> int { return value_; }
  auto operator++() noexcept -> rank& { ++value_; return *this; }
  auto operator--() noexcept -> rank& { --value_; return *this; }
  auto operator++(int) noexcept -> rank { auto r = *this; ++value_; return r; }
  auto operator+=(int d) noexcept -> rank& { value_ += d; return *this; }
  auto operator-=(int d) noexcept -> rank& { value_ -= d; return *this; }
  friend constexpr auto operator==(rank a, rank b) noexcept -> bool { return a.value_ == b.value_; }
  friend constexpr auto operator!=(rank a, rank b) noexcept -> bool { return a.value_ != b.value_; }
  friend constexpr auto operator<(rank a, rank b) noexcept -> bool { return a.value_ < b.value_; }
  friend constexpr auto operator>(rank a, rank b) noexcept -> bool { return a.value_ > b.value_; }
  friend constexpr auto operator<=(rank a, rank b) noexcept -> bool { return a.value_ <= b.value_; }
  friend constexpr auto operator>=(rank a, rank b) noexcept -> bool { return a.value_ >= b.value_; }
  friend constexpr auto operator+(rank a, int d) noexcept -> rank { return rank{a.value_ + d}; }
  friend constexpr auto operator-(rank a, int d) noexcept -> rank { return rank{a.value_ - d}; }
  friend constexpr auto operator-(rank a, rank b) noexcept -> int { return a.value_ - b.value_; }
};

constexpr rank null_process{-1};
constexpr rank any_source{-2};

struct tag {
  int value = 0;
  constexpr tag() noexcept = default;
  constexpr explicit tag(int v) noexcept : value{v} {}
};
struct color {
  int value = 0;
  constexpr color() noexcept = default;
  constexpr explicit color(int v) noexcept : value{v} {}
};
struct count {
  int value = 0;
  constexpr count() noexcept = default;
  constexpr explicit count(int v) noexcept : value{v} {}
  template <typename Integer, typename = std::enable_if_t<std::is_integral<Integer>::value>>
  constexpr explicit count(Integer v) noexcept : value{static_cast<int>(v)} {}
};

namespace tags {
struct world_communicator_t {};
constexpr world_communicator_t world_communicator{};
struct plus_t {};
constexpr plus_t plus{};
}  // namespace tags
using plus_t = tags::plus_t;

struct in_place_t {};
constexpr in_place_t in_place{};
struct ignore_status_t {};
constexpr ignore_status_t ignore_status{};

class status {};

class communicator {
 public:
  communicator() noexcept = default;
  explicit communicator(tags::world_communicator_t) noexcept {}
  communicator(communicator const&, color, int, environment const&) noexcept {}
  auto rank(environment const&) const noexcept -> yampi::rank { return yampi::rank{0}; }
  auto size(environment const&) const noexcept -> int { return 1; }
};

class intercommunicator {
 public:
  intercommunicator() noexcept = default;
  auto rank(environment const&) const noexcept -> yampi::rank { return yampi::rank{0}; }
  auto size(environment const&) const noexcept -> int { return 1; }
  auto remote_size(environment const&) const noexcept -> int { return 1; }
};

struct message_envelope {
  yampi::rank source, destination;
  message_envelope(yampi::rank s, yampi::rank d, communicator const&) noexcept : source{s}, destination{d} {}
};

// Datatypes carry no information in one process.
template <typename Derived>
class datatype_base {};
class datatype : public datatype_base<datatype> {
 public:
  datatype() noexcept = default;
  template <typename... Args>
  explicit datatype(Args const&...) noexcept {}
};
template <typename T>
class predefined_datatype : public datatype_base<predefined_datatype<T>> {};

struct fixed_blocks {
  template <typename... Args>
  explicit fixed_blocks(Args const&...) noexcept {}
};

// A buffer is a contiguous run of values.
template <typename T>
class buffer {
  T* data_;
  std::size_t count_;

 public:
  buffer(T* data, std::size_t count) noexcept : data_{data}, count_{count} {}
  auto data() const noexcept -> T* { return data_; }
  auto count() const noexcept -> std::size_t { return count_; }
  auto begin() const noexcept -> T* { return data_; }
  auto end() const noexcept -> T* { return data_ + count_; }
};

template <typename T>
auto make_buffer(T& value) -> buffer<T> { return {std::addressof(value), 1u}; }
template <typename T, typename Derived>
auto make_buffer(T& value, datatype_base<Derived> const&) -> buffer<T> { return {std::addressof(value), 1u}; }
template <typename T, typename Derived>
auto make_buffer(T const& value, datatype_base<Derived> const&) -> buffer<T const> { return {std::addressof(value), 1u}; }
template <typename Iterator, typename = decltype(*std::declval<Iterator>())>
auto make_buffer(Iterator first, Iterator last)
{
  using T = std::remove_reference_t<decltype(*first)>;
  return buffer<T>{std::addressof(*first), static_cast<std::size_t>(last - first)};
}
template <typename Iterator, typename Derived>
auto make_buffer(Iterator first, Iterator last, datatype_base<Derived> const&)
{
  return make_buffer(first, last);
}
template <typename Range>
auto range_to_buffer(Range& range)
{
  using std::begin;
  using std::end;
  return make_buffer(begin(range), end(range));
}
template <typename Range, typename Derived>
auto range_to_buffer(Range& range, datatype_base<Derived> const&)
{
  return range_to_buffer(range);
}

class binary_operation {
 public:
  explicit binary_operation(tags::plus_t) noexcept {}
};

namespace one_process_detail {
template <typename T, typename OutputIterator>
void copy_out(buffer<T> const& send, OutputIterator out)
{
  std::copy(send.begin(), send.end(), out);
}
[[noreturn]] inline void several_processes(char const* what)
{
  throw std::logic_error(std::string{"yampi stand-in (one process): "} + what + " needs several processes");
}
}  // namespace one_process_detail

// Collectives over one rank.
template <typename T, typename Comm>
void all_reduce(in_place_t, buffer<T> const&, binary_operation const&, Comm const&, environment const&) {}
template <typename T, typename OutputIterator, typename Comm>
void all_reduce(buffer<T> const& send, OutputIterator out, binary_operation const&, Comm const&, environment const&)
{
  one_process_detail::copy_out(send, out);
}
template <typename T, typename Comm>
void reduce(in_place_t, buffer<T> const&, binary_operation const&, yampi::rank, Comm const&, environment const&) {}
template <typename T, typename OutputIterator, typename Comm>
void reduce(buffer<T> const& send, OutputIterator out, binary_operation const&, yampi::rank, Comm const&,
            environment const&)
{
  one_process_detail::copy_out(send, out);
}
template <typename T, typename Comm>
void broadcast(buffer<T> const&, yampi::rank, Comm const&, environment const&) {}
template <typename T, typename OutputIterator, typename Comm>
void gather(buffer<T> const& send, OutputIterator out, yampi::rank, Comm const&, environment const&)
{
  one_process_detail::copy_out(send, out);
}
template <typename T, typename Comm>
void barrier(Comm const&, environment const&) {}
inline void barrier(communicator const&, environment const&) {}

// A send/receive between rank 0 and itself: the send buffer lands in the
// receive buffer.  Any other partner does not exist in one process.
template <typename S, typename R, typename Comm>
void send_receive(ignore_status_t, buffer<S> const& send, yampi::rank dest, tag, buffer<R> const& recv,
                  yampi::rank source, tag, Comm const&, environment const&)
{
  if (dest != yampi::rank{0} || source != yampi::rank{0} || recv.count() != send.count())
    one_process_detail::several_processes("send_receive with another rank");
  std::copy(send.begin(), send.end(), recv.begin());
}
template <typename T, typename Comm>
void send_receive(ignore_status_t, buffer<T> const& buf, yampi::rank dest, tag, yampi::rank source, tag, Comm const&,
                  environment const&)
{
  if (dest != yampi::rank{0} || source != yampi::rank{0})
    one_process_detail::several_processes("send_receive with another rank");
  (void)buf;
}
template <typename T, typename Comm>
void send(buffer<T> const&, yampi::rank, tag, Comm const&, environment const&)
{
  one_process_detail::several_processes("send");
}
template <typename T, typename Comm>
void receive(ignore_status_t, buffer<T> const&, yampi::rank, tag, Comm const&, environment const&)
{
  one_process_detail::several_processes("receive");
}

// An all-to-all over one rank leaves the data in place.
template <typename T, typename Comm>
void complete_exchange(in_place_t, buffer<T> const&, Comm const&, environment const&) {}
template <typename... Args>
void noncontiguous_complete_exchange(Args const&...)
{
  one_process_detail::several_processes("noncontiguous_complete_exchange");
}
template <typename... Args>
int make_noncontiguous_buffer(Args const&...)
{
  return 0;
}

// The lowest rank that can do I/O, as an optional rank: always rank 0 here.
struct io_process {
  yampi::rank value{0};
  explicit operator bool() const noexcept { return true; }
  auto operator*() const noexcept -> yampi::rank { return value; }
};
inline auto lowest_io_process(environment const&) -> io_process { return io_process{}; }

struct wall_clock {
  using duration = std::chrono::duration<double>;
  using time_point = std::chrono::time_point<std::chrono::steady_clock, duration>;
  static auto now(environment const&) -> time_point { return std::chrono::steady_clock::now(); }
};

namespace algorithm {
// Exchanges of data blocks with a partner rank: reached only for global qubits.
template <typename... Args>
void swap(Args&&...)
{
  one_process_detail::several_processes("algorithm::swap");
}
template <typename... Args>
void transform(Args&&...)
{
  one_process_detail::several_processes("algorithm::transform");
}
}  // namespace algorithm

}  // namespace yampi

#endif
