// Project-written stand-in for boost::iterator_range / make_iterator_range as
// used by the reference's ket headers.  Used to build the reference's code in this image, which has no Boost.
#ifndef RBK_SHIM_BOOST_RANGE_ITERATOR_RANGE_HPP
#define RBK_SHIM_BOOST_RANGE_ITERATOR_RANGE_HPP

#include <cstddef>
#include <iterator>
#include <utility>

namespace boost {

template <typename Iterator>
class iterator_range
{
 public:
  using iterator = Iterator;
  using const_iterator = Iterator;
  using value_type = typename std::iterator_traits<Iterator>::value_type;
  using reference = typename std::iterator_traits<Iterator>::reference;
  using difference_type = typename std::iterator_traits<Iterator>::difference_type;
  using size_type = std::size_t;

  iterator_range() = default;
  iterator_range(Iterator first, Iterator last) : first_(first), last_(last) { }
  template <typename Range>
  explicit iterator_range(Range& range) : first_(std::begin(range)), last_(std::end(range)) { }

  Iterator begin() const { return first_; }
  Iterator end() const { return last_; }
  bool empty() const { return first_ == last_; }
  size_type size() const { return static_cast<size_type>(std::distance(first_, last_)); }
  reference front() const { return *first_; }
  reference operator[](difference_type n) const { return first_[n]; }

 private:
  Iterator first_{};
  Iterator last_{};
};

template <typename Iterator>
inline iterator_range<Iterator> make_iterator_range(Iterator first, Iterator last)
{ return iterator_range<Iterator>(first, last); }

template <typename Range>
inline auto make_iterator_range(Range& range) -> iterator_range<decltype(std::begin(range))>
{ return iterator_range<decltype(std::begin(range))>(std::begin(range), std::end(range)); }

template <typename Range>
inline auto make_iterator_range(Range const& range) -> iterator_range<decltype(std::begin(range))>
{ return iterator_range<decltype(std::begin(range))>(std::begin(range), std::end(range)); }

template <typename Iterator, typename Size>
inline iterator_range<Iterator> make_iterator_range_n(Iterator first, Size n)
{ return iterator_range<Iterator>(first, std::next(first, n)); }

// Kept out of argument-dependent lookup (like Boost does) so that
// `using std::begin; begin(r)` in the reference stays unambiguous.
namespace range_adl_barrier {
template <typename Range>
inline auto size(Range const& range) -> std::size_t
{ return static_cast<std::size_t>(std::distance(std::begin(range), std::end(range))); }

template <typename Range>
inline auto begin(Range& range) -> decltype(std::begin(range)) { return std::begin(range); }
template <typename Range>
inline auto begin(Range const& range) -> decltype(std::begin(range)) { return std::begin(range); }
template <typename Range>
inline auto end(Range& range) -> decltype(std::end(range)) { return std::end(range); }
template <typename Range>
inline auto end(Range const& range) -> decltype(std::end(range)) { return std::end(range); }

} // namespace range_adl_barrier
using namespace range_adl_barrier;

} // namespace boost

#endif
