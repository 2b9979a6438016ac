// Project-written stand-in for fmt::format as bra uses it (the spin table of
// DO MEASUREMENT, bra/src/state.cpp): automatic argument indexing and the
// format spec [[fill]align][sign][width][.precision][type] for strings,
// integers and floating-point values (types s, d, f, e, g; none).  Alignment
// follows fmt: strings to the left, numbers to the right, '^' centred with the
// odd padding character on the right.  Used to build the reference's code in
// this image, which does not have fmt.
#ifndef RBK_SHIM_FMT_CORE_H
#define RBK_SHIM_FMT_CORE_H

#include <cstdio>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace fmt {

struct format_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

namespace detail {

struct spec {
  char fill = ' ';
  char align = 0;  // '<', '>', '^' or 0 (the type's default)
  char sign = '-';
  int width = 0;
  int precision = -1;
  char type = 0;
};

inline spec parse_spec(std::string const& s)
{
  spec r;
  size_t i = 0;
  auto is_align = [](char c) { return c == '<' || c == '>' || c == '^'; };
  if (s.size() >= 2 && is_align(s[1])) { r.fill = s[0]; r.align = s[1]; i = 2; }
  else if (!s.empty() && is_align(s[0])) { r.align = s[0]; i = 1; }
  if (i < s.size() && (s[i] == '+' || s[i] == '-' || s[i] == ' ')) r.sign = s[i++];
  while (i < s.size() && s[i] >= '0' && s[i] <= '9') r.width = r.width * 10 + (s[i++] - '0');
  if (i < s.size() && s[i] == '.') {
    ++i;
    r.precision = 0;
    while (i < s.size() && s[i] >= '0' && s[i] <= '9') r.precision = r.precision * 10 + (s[i++] - '0');
  }
  if (i < s.size()) r.type = s[i++];
  if (i != s.size()) throw format_error("invalid format specifier: " + s);
  return r;
}

inline std::string pad(std::string body, spec const& sp, char default_align)
{
  const int n = static_cast<int>(body.size());
  if (sp.width <= n) return body;
  const int padding = sp.width - n;
  const char align = sp.align ? sp.align : default_align;
  int left = 0;
  if (align == '>') left = padding;
  else if (align == '^') left = padding / 2;
  return std::string(static_cast<size_t>(left), sp.fill) + body + std::string(static_cast<size_t>(padding - left), sp.fill);
}

inline std::string format_arg(spec const& sp, std::string const& v)
{
  std::string body = sp.precision >= 0 ? v.substr(0, static_cast<size_t>(sp.precision)) : v;
  return pad(body, sp, '<');
}
inline std::string format_arg(spec const& sp, const char* v) { return format_arg(sp, std::string(v)); }

template <typename T>
inline typename std::enable_if<std::is_floating_point<T>::value, std::string>::type format_arg(spec const& sp, T v)
{
  char conv = sp.type ? sp.type : 'g';
  std::string f = "%";
  if (sp.sign == '+') f += '+';
  else if (sp.sign == ' ') f += ' ';
  if (sp.precision >= 0) f += "." + std::to_string(sp.precision);
  else if (!sp.type) { f += ".17"; }
  f += conv;
  char buf[512];
  std::snprintf(buf, sizeof(buf), f.c_str(), static_cast<double>(v));
  return pad(buf, sp, '>');
}

template <typename T>
inline typename std::enable_if<std::is_integral<T>::value, std::string>::type format_arg(spec const& sp, T v)
{
  std::string body = std::to_string(v);
  if (v >= 0 && sp.sign == '+') body = "+" + body;
  else if (v >= 0 && sp.sign == ' ') body = " " + body;
  return pad(body, sp, '>');
}

inline void format_rest(std::string& out, std::string const& f, size_t pos)
{
  for (size_t i = pos; i < f.size(); ++i) {
    if (f[i] == '{' && i + 1 < f.size() && f[i + 1] == '{') { out += '{'; ++i; }
    else if (f[i] == '}' && i + 1 < f.size() && f[i + 1] == '}') { out += '}'; ++i; }
    else if (f[i] == '{') throw format_error("argument index out of range");
    else out += f[i];
  }
}

template <typename T, typename... Rest>
inline void format_rest(std::string& out, std::string const& f, size_t pos, T const& v, Rest const&... rest)
{
  for (size_t i = pos; i < f.size(); ++i) {
    if (f[i] == '{' && i + 1 < f.size() && f[i + 1] == '{') { out += '{'; ++i; continue; }
    if (f[i] == '}' && i + 1 < f.size() && f[i + 1] == '}') { out += '}'; ++i; continue; }
    if (f[i] != '{') { out += f[i]; continue; }
    const size_t close = f.find('}', i);
    if (close == std::string::npos) throw format_error("unmatched '{' in format string");
    std::string field = f.substr(i + 1, close - i - 1);
    const size_t colon = field.find(':');
    if (colon != std::string::npos) field = field.substr(colon + 1);
    else field.clear();
    out += format_arg(parse_spec(field), v);
    format_rest(out, f, close + 1, rest...);
    return;
  }
}

}  // namespace detail

template <typename... Args>
inline std::string format(std::string const& f, Args const&... args)
{
  std::string out;
  detail::format_rest(out, f, 0, args...);
  return out;
}

}  // namespace fmt

#endif
