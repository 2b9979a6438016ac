// Project-written stand-in for boost::variant, boost::get and
// boost::apply_visitor as bra uses them (parameters that are a number or a
// variable name, bra/include/bra/interpreter.hpp, bra/src/*.cpp), on
// std::variant.  As in Boost, a value converts to the alternative that plain
// overload resolution picks, narrowing included (a double assigned to
// variant<int, std::string> becomes the int), where std::variant refuses
// narrowing.  bra relies on that, and on lexical_cast arriving with these
// headers.  Used to build the reference's code in this image, which has no
// Boost.
#ifndef RBK_SHIM_BOOST_VARIANT_VARIANT_HPP
#define RBK_SHIM_BOOST_VARIANT_VARIANT_HPP

#include <exception>
#include <type_traits>
#include <utility>
#include <variant>

#include <boost/lexical_cast.hpp>
#include <boost/variant/static_visitor.hpp>

namespace boost {

namespace variant_detail {
template <std::size_t I, typename T>
struct one { static std::integral_constant<std::size_t, I> pick(T); };
template <typename Seq, typename... Ts>
struct overloads;
template <std::size_t... Is, typename... Ts>
struct overloads<std::index_sequence<Is...>, Ts...> : one<Is, Ts>... { using one<Is, Ts>::pick...; };
// Index of the alternative that overload resolution picks for a U.
template <typename U, typename... Ts>
using pick_t = decltype(overloads<std::index_sequence_for<Ts...>, Ts...>::pick(std::declval<U>()));
}  // namespace variant_detail

struct bad_get : std::exception {
  const char* what() const noexcept override { return "boost::bad_get: the variant holds another type"; }
};

template <typename... Ts>
class variant : public std::variant<Ts...>
{
  using base = std::variant<Ts...>;

 public:
  variant() = default;
  variant(variant const&) = default;
  variant(variant&&) = default;
  variant& operator=(variant const&) = default;
  variant& operator=(variant&&) = default;

  template <typename U, typename D = typename std::decay<U>::type,
            typename = typename std::enable_if<!std::is_same<D, variant>::value && !std::is_same<D, base>::value>::type,
            std::size_t I = variant_detail::pick_t<U, Ts...>::value>
  variant(U&& u) : base(std::in_place_index<I>, std::forward<U>(u)) { }

  template <typename U, typename D = typename std::decay<U>::type,
            typename = typename std::enable_if<!std::is_same<D, variant>::value && !std::is_same<D, base>::value>::type,
            std::size_t I = variant_detail::pick_t<U, Ts...>::value>
  variant& operator=(U&& u)
  {
    this->base::template emplace<I>(std::forward<U>(u));
    return *this;
  }

  int which() const noexcept { return static_cast<int>(this->index()); }
  bool empty() const noexcept { return false; }
  base& as_std() noexcept { return *this; }
  base const& as_std() const noexcept { return *this; }
};

template <typename T, typename... Ts>
inline T* get(variant<Ts...>* v) noexcept { return v ? std::get_if<T>(&v->as_std()) : nullptr; }
template <typename T, typename... Ts>
inline T const* get(variant<Ts...> const* v) noexcept { return v ? std::get_if<T>(&v->as_std()) : nullptr; }
template <typename T, typename... Ts>
inline T& get(variant<Ts...>& v)
{
  if (T* p = std::get_if<T>(&v.as_std())) return *p;
  throw bad_get{};
}
template <typename T, typename... Ts>
inline T const& get(variant<Ts...> const& v)
{
  if (T const* p = std::get_if<T>(&v.as_std())) return *p;
  throw bad_get{};
}

template <typename Visitor, typename... Ts>
inline decltype(auto) apply_visitor(Visitor&& visitor, variant<Ts...>& v)
{ return std::visit(std::forward<Visitor>(visitor), v.as_std()); }
template <typename Visitor, typename... Ts>
inline decltype(auto) apply_visitor(Visitor&& visitor, variant<Ts...> const& v)
{ return std::visit(std::forward<Visitor>(visitor), v.as_std()); }
template <typename Visitor, typename... Ts>
inline decltype(auto) apply_visitor(Visitor&& visitor, variant<Ts...>&& v)
{ return std::visit(std::forward<Visitor>(visitor), std::move(v.as_std())); }

}  // namespace boost

#endif
