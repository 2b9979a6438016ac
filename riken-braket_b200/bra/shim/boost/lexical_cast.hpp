// Project-written stand-in for boost::lexical_cast as bra's interpreter uses
// it: numbers read from, and written to, strings.  A conversion must consume
// the whole input (no leading or trailing characters, whitespace included);
// floating-point values are written with enough digits to read back the same
// value.  Used to build the reference's code in this image, which has no Boost.
#ifndef RBK_SHIM_BOOST_LEXICAL_CAST_HPP
#define RBK_SHIM_BOOST_LEXICAL_CAST_HPP

#include <ios>
#include <limits>
#include <sstream>
#include <string>
#include <type_traits>
#include <typeinfo>

namespace boost {

struct bad_lexical_cast : std::bad_cast {
  const char* what() const noexcept override { return "bad lexical cast: source type value could not be interpreted as target"; }
};

namespace lexical_cast_detail {
template <typename S>
inline void put(std::ostringstream& os, S const& s)
{
  if constexpr (std::is_floating_point<S>::value) os.precision(std::numeric_limits<S>::max_digits10);
  os << s;
}
}  // namespace lexical_cast_detail

template <typename T, typename S>
inline T lexical_cast(S const& source)
{
  std::ostringstream os;
  lexical_cast_detail::put(os, source);
  if constexpr (std::is_same<T, std::string>::value) {
    return os.str();
  } else {
    std::istringstream is(os.str());
    is >> std::noskipws;
    T value{};
    if constexpr (std::is_same<T, char>::value || std::is_same<T, signed char>::value || std::is_same<T, unsigned char>::value) {
      if (os.str().size() != 1) throw bad_lexical_cast{};
      value = static_cast<T>(os.str()[0]);
      return value;
    } else {
      if (!(is >> value)) throw bad_lexical_cast{};
      if (is.peek() != std::char_traits<char>::eof()) throw bad_lexical_cast{};
      return value;
    }
  }
}

}  // namespace boost

#endif
