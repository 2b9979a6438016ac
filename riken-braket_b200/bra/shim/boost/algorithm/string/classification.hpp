// Project-written stand-in for boost::algorithm::is_space / is_any_of
// (character predicates for split and trim).  Used to build the reference's
// code in this image, which has no Boost.
#ifndef RBK_SHIM_BOOST_ALGORITHM_STRING_CLASSIFICATION_HPP
#define RBK_SHIM_BOOST_ALGORITHM_STRING_CLASSIFICATION_HPP
#include <cctype>
#include <string>
namespace boost {
namespace algorithm {
struct is_space_pred {
  bool operator()(char c) const { return std::isspace(static_cast<unsigned char>(c)) != 0; }
};
inline is_space_pred is_space() { return {}; }
struct is_any_of_pred {
  std::string set;
  bool operator()(char c) const { return set.find(c) != std::string::npos; }
};
inline is_any_of_pred is_any_of(std::string const& set) { return {set}; }
}  // namespace algorithm
using algorithm::is_any_of;
using algorithm::is_space;
}  // namespace boost
#endif
