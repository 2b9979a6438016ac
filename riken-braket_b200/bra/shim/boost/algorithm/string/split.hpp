// Project-written stand-in for boost::algorithm::split into a container of
// std::string, with token_compress_on / _off: with compression, adjacent
// separators make one; without, every separator ends a (possibly empty) token.
// Used to build the reference's code in this image, which has no Boost.
#ifndef RBK_SHIM_BOOST_ALGORITHM_STRING_SPLIT_HPP
#define RBK_SHIM_BOOST_ALGORITHM_STRING_SPLIT_HPP
#include <string>
#include <boost/algorithm/string/classification.hpp>
namespace boost {
namespace algorithm {
enum token_compress_mode_type { token_compress_on, token_compress_off };
template <typename Container, typename Predicate>
inline Container& split(Container& out, std::string const& input, Predicate is_separator,
                        token_compress_mode_type mode = token_compress_off)
{
  out.clear();
  std::string token;
  bool last_was_separator = false;
  for (char c : input) {
    if (is_separator(c)) {
      if (mode == token_compress_on && last_was_separator) continue;
      out.push_back(token);
      token.clear();
      last_was_separator = true;
    } else {
      token.push_back(c);
      last_was_separator = false;
    }
  }
  out.push_back(token);
  return out;
}
}  // namespace algorithm
using algorithm::split;
using algorithm::token_compress_mode_type;
using algorithm::token_compress_off;
using algorithm::token_compress_on;
}  // namespace boost
#endif
