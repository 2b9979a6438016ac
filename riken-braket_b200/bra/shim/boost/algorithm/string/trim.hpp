// Project-written stand-in for boost::algorithm::trim / trim_copy (whitespace
// of the classic locale).  Used to build the reference's code in this image,
// which has no Boost.
#ifndef RBK_SHIM_BOOST_ALGORITHM_STRING_TRIM_HPP
#define RBK_SHIM_BOOST_ALGORITHM_STRING_TRIM_HPP
#include <cctype>
#include <string>
namespace boost {
namespace algorithm {
inline void trim_left(std::string& s)
{
  std::string::size_type i = 0;
  while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
  s.erase(0, i);
}
inline void trim_right(std::string& s)
{
  std::string::size_type n = s.size();
  while (n > 0 && std::isspace(static_cast<unsigned char>(s[n - 1]))) --n;
  s.erase(n);
}
inline void trim(std::string& s) { trim_right(s); trim_left(s); }
inline std::string trim_copy(std::string s) { trim(s); return s; }
}  // namespace algorithm
using algorithm::trim;
using algorithm::trim_copy;
using algorithm::trim_left;
using algorithm::trim_right;
}  // namespace boost
#endif
