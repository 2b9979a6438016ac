// Project-written stand-in.  Test infrastructure only.
#ifndef RBK_SHIM_BOOST_IS_NOTHROW_SWAPPABLE_HPP
#define RBK_SHIM_BOOST_IS_NOTHROW_SWAPPABLE_HPP
#include <type_traits>
namespace boost { template <typename T> using is_nothrow_swappable = std::is_nothrow_swappable<T>; }
#endif
