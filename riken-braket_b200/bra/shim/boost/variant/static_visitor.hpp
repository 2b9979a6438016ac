// Project-written stand-in for boost::static_visitor (see variant.hpp).
#ifndef RBK_SHIM_BOOST_VARIANT_STATIC_VISITOR_HPP
#define RBK_SHIM_BOOST_VARIANT_STATIC_VISITOR_HPP
namespace boost {
template <typename R = void>
struct static_visitor {
  using result_type = R;
};
}  // namespace boost
#endif
