// Project-written stand-in for boost::algorithm::to_upper / to_upper_copy /
// to_lower / to_lower_copy on std::string (ASCII, the classic locale, as bra's
// mnemonics are).  Used to build the reference's code in this image, which
// has no Boost.
#ifndef RBK_SHIM_BOOST_ALGORITHM_STRING_CASE_CONV_HPP
#define RBK_SHIM_BOOST_ALGORITHM_STRING_CASE_CONV_HPP
#include <cctype>
#include <string>
namespace boost {
namespace algorithm {
inline void to_upper(std::string& s) { for (char& c : s) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c))); }
inline void to_lower(std::string& s) { for (char& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c))); }
inline std::string to_upper_copy(std::string s) { to_upper(s); return s; }
inline std::string to_lower_copy(std::string s) { to_lower(s); return s; }
}  // namespace algorithm
using algorithm::to_lower;
using algorithm::to_lower_copy;
using algorithm::to_upper;
using algorithm::to_upper_copy;
}  // namespace boost
#endif
