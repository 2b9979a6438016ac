// Project-written stand-in for `range | boost::adaptors::transformed(f)` as used
// by the reference's ket headers (e.g. ket/include/ket/gate/phase_shift.hpp:2034).
// Random-access only, which is all the reference needs.  Used to build the reference's code in this image, which has no Boost.
#ifndef RBK_SHIM_BOOST_RANGE_ADAPTOR_TRANSFORMED_HPP
#define RBK_SHIM_BOOST_RANGE_ADAPTOR_TRANSFORMED_HPP

#include <cstddef>
#include <iterator>
#include <optional>
#include <type_traits>
#include <utility>
#include <boost/range/iterator_range.hpp>

namespace boost {
namespace range_shim_detail {

template <typename Iterator, typename Function>
class transform_iterator
{
 public:
  using iterator_category = std::random_access_iterator_tag;
  using reference = decltype(std::declval<Function const&>()(*std::declval<Iterator>()));
  using value_type = typename std::decay<reference>::type;
  using difference_type = typename std::iterator_traits<Iterator>::difference_type;
  using pointer = void;

  transform_iterator() = default;
  transform_iterator(Iterator it, Function const& f) : it_(it) { f_.emplace(f); }
  transform_iterator(transform_iterator const& other) : it_(other.it_)
  { if (other.f_) f_.emplace(*other.f_); }
  transform_iterator& operator=(transform_iterator const& other)
  {
    it_ = other.it_;
    f_.reset();
    if (other.f_) f_.emplace(*other.f_);
    return *this;
  }

  reference operator*() const { return (*f_)(*it_); }
  reference operator[](difference_type n) const { return (*f_)(it_[n]); }
  transform_iterator& operator++() { ++it_; return *this; }
  transform_iterator operator++(int) { auto t = *this; ++it_; return t; }
  transform_iterator& operator--() { --it_; return *this; }
  transform_iterator operator--(int) { auto t = *this; --it_; return t; }
  transform_iterator& operator+=(difference_type n) { it_ += n; return *this; }
  transform_iterator& operator-=(difference_type n) { it_ -= n; return *this; }
  friend transform_iterator operator+(transform_iterator t, difference_type n) { t += n; return t; }
  friend transform_iterator operator+(difference_type n, transform_iterator t) { t += n; return t; }
  friend transform_iterator operator-(transform_iterator t, difference_type n) { t -= n; return t; }
  friend difference_type operator-(transform_iterator const& a, transform_iterator const& b) { return a.it_ - b.it_; }
  friend bool operator==(transform_iterator const& a, transform_iterator const& b) { return a.it_ == b.it_; }
  friend bool operator!=(transform_iterator const& a, transform_iterator const& b) { return a.it_ != b.it_; }
  friend bool operator<(transform_iterator const& a, transform_iterator const& b) { return a.it_ < b.it_; }
  friend bool operator>(transform_iterator const& a, transform_iterator const& b) { return a.it_ > b.it_; }
  friend bool operator<=(transform_iterator const& a, transform_iterator const& b) { return a.it_ <= b.it_; }
  friend bool operator>=(transform_iterator const& a, transform_iterator const& b) { return a.it_ >= b.it_; }

 private:
  Iterator it_{};
  std::optional<Function> f_{};
};

template <typename Function>
struct transform_holder { Function f; };

// Found by argument-dependent lookup through transform_holder.
template <typename Range, typename Function>
inline auto operator|(Range const& range, transform_holder<Function> const& holder)
  -> iterator_range<transform_iterator<decltype(std::begin(range)), Function>>
{
  using it = transform_iterator<decltype(std::begin(range)), Function>;
  return iterator_range<it>(it(std::begin(range), holder.f), it(std::end(range), holder.f));
}

} // namespace range_shim_detail

namespace adaptors {
template <typename Function>
inline range_shim_detail::transform_holder<Function> transformed(Function f)
{ return range_shim_detail::transform_holder<Function>{f}; }
} // namespace adaptors

} // namespace boost

#endif
