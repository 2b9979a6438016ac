// Project-written stand-in: boost::empty for ranges.
#ifndef RBK_SHIM_BOOST_RANGE_EMPTY_HPP
#define RBK_SHIM_BOOST_RANGE_EMPTY_HPP
#include <iterator>
#include <boost/range/iterator_range.hpp>
namespace boost {
namespace range_adl_barrier {
template <typename Range>
inline bool empty(Range const& range) { return std::begin(range) == std::end(range); }
}  // namespace range_adl_barrier
}  // namespace boost
#endif
