// Project-written stand-in for boost::optional / boost::none as used by the
// reference (ket/include/ket/utility/parallel/loop_n.hpp:167, bra fused gates).
// Used to build the reference's code in this image, which has no Boost.
#ifndef RBK_SHIM_BOOST_OPTIONAL_HPP
#define RBK_SHIM_BOOST_OPTIONAL_HPP
#include <optional>
namespace boost {
template <typename T>
using optional = std::optional<T>;
constexpr std::nullopt_t none = std::nullopt;
}
#endif
