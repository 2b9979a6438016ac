// Project-written stand-in: boost::sub_range as an iterator_range.  Used to build the reference's code in this image, which has no Boost.
#ifndef RBK_SHIM_BOOST_RANGE_SUB_RANGE_HPP
#define RBK_SHIM_BOOST_RANGE_SUB_RANGE_HPP
#include <boost/range/iterator_range.hpp>
namespace boost {
template <typename Range>
using sub_range = iterator_range<decltype(std::begin(std::declval<Range&>()))>;
}
#endif
