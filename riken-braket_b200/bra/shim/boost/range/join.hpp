// Project-written stand-in for boost::join over two random-access ranges with
// the same value type, as used by the reference's ket headers (e.g.
// ket/include/ket/gate/phase_shift.hpp:2032).  Elements are yielded by value.
// Used to build the reference's code in this image, which has no Boost.
#ifndef RBK_SHIM_BOOST_RANGE_JOIN_HPP
#define RBK_SHIM_BOOST_RANGE_JOIN_HPP

#include <cstddef>
#include <iterator>
#include <type_traits>
#include <boost/range/iterator_range.hpp>

namespace boost {
namespace range_shim_detail {

template <typename Iterator1, typename Iterator2>
class join_iterator
{
 public:
  using iterator_category = std::random_access_iterator_tag;
  using value_type = typename std::decay<decltype(*std::declval<Iterator1>())>::type;
  using reference = value_type;
  using difference_type = std::ptrdiff_t;
  using pointer = void;

  join_iterator() = default;
  join_iterator(Iterator1 first1, difference_type size1, Iterator2 first2, difference_type pos)
    : first1_(first1), first2_(first2), size1_(size1), pos_(pos) { }

  reference operator*() const { return (*this)[0]; }
  reference operator[](difference_type n) const
  {
    auto const p = pos_ + n;
    if (p < size1_) return static_cast<value_type>(first1_[p]);
    return static_cast<value_type>(first2_[p - size1_]);
  }
  join_iterator& operator++() { ++pos_; return *this; }
  join_iterator operator++(int) { auto t = *this; ++pos_; return t; }
  join_iterator& operator--() { --pos_; return *this; }
  join_iterator operator--(int) { auto t = *this; --pos_; return t; }
  join_iterator& operator+=(difference_type n) { pos_ += n; return *this; }
  join_iterator& operator-=(difference_type n) { pos_ -= n; return *this; }
  friend join_iterator operator+(join_iterator t, difference_type n) { t += n; return t; }
  friend join_iterator operator+(difference_type n, join_iterator t) { t += n; return t; }
  friend join_iterator operator-(join_iterator t, difference_type n) { t -= n; return t; }
  friend difference_type operator-(join_iterator const& a, join_iterator const& b) { return a.pos_ - b.pos_; }
  friend bool operator==(join_iterator const& a, join_iterator const& b) { return a.pos_ == b.pos_; }
  friend bool operator!=(join_iterator const& a, join_iterator const& b) { return a.pos_ != b.pos_; }
  friend bool operator<(join_iterator const& a, join_iterator const& b) { return a.pos_ < b.pos_; }
  friend bool operator>(join_iterator const& a, join_iterator const& b) { return a.pos_ > b.pos_; }
  friend bool operator<=(join_iterator const& a, join_iterator const& b) { return a.pos_ <= b.pos_; }
  friend bool operator>=(join_iterator const& a, join_iterator const& b) { return a.pos_ >= b.pos_; }

 private:
  Iterator1 first1_{};
  Iterator2 first2_{};
  difference_type size1_ = 0;
  difference_type pos_ = 0;
};

} // namespace range_shim_detail

template <typename Range1, typename Range2>
inline auto join(Range1 const& range1, Range2 const& range2)
  -> iterator_range<range_shim_detail::join_iterator<decltype(std::begin(range1)), decltype(std::begin(range2))>>
{
  using it = range_shim_detail::join_iterator<decltype(std::begin(range1)), decltype(std::begin(range2))>;
  auto const size1 = static_cast<std::ptrdiff_t>(std::distance(std::begin(range1), std::end(range1)));
  auto const size2 = static_cast<std::ptrdiff_t>(std::distance(std::begin(range2), std::end(range2)));
  return iterator_range<it>(
    it(std::begin(range1), size1, std::begin(range2), 0),
    it(std::begin(range1), size1, std::begin(range2), size1 + size2));
}

} // namespace boost

#endif
