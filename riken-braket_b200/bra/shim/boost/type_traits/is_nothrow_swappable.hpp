// Project-written stand-in for boost::is_nothrow_swappable (used by the
// reference's ket::mpi headers before C++17).  Used to build the reference's code in this image, which has no Boost.
#ifndef RBK_SHIM_BOOST_IS_NOTHROW_SWAPPABLE_HPP
#define RBK_SHIM_BOOST_IS_NOTHROW_SWAPPABLE_HPP
#include <type_traits>
#include <utility>
namespace boost {
namespace rbk_shim_detail {
using std::swap;
template <typename T>
struct nothrow_swap : std::integral_constant<bool, noexcept(swap(std::declval<T&>(), std::declval<T&>()))> {};
}  // namespace rbk_shim_detail
template <typename T>
struct is_nothrow_swappable : rbk_shim_detail::nothrow_swap<T> {};
}  // namespace boost
#endif
