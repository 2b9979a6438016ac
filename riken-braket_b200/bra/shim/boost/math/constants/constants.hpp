// Project-written stand-in for the few Boost.Math constants the reference's
// ket headers use (ket/include/ket/gate/hadamard.hpp, phase_shift.hpp, ...).
// Test infrastructure only: lets the oracle compile the reference's own
// header-only gate code without Boost.  Each value is a decimal literal of the
// target type, so the compiler rounds it correctly (the Boost values are the
// correctly rounded constants too).
#ifndef RBK_SHIM_BOOST_MATH_CONSTANTS_HPP
#define RBK_SHIM_BOOST_MATH_CONSTANTS_HPP

namespace boost { namespace math { namespace constants {

#define RBK_SHIM_CONSTANT(name, digits)                                          \
  template <typename T> constexpr T name();                                      \
  template <> constexpr float name<float>() { return digits##f; }                \
  template <> constexpr double name<double>() { return digits; }                 \
  template <> constexpr long double name<long double>() { return digits##L; }

RBK_SHIM_CONSTANT(half, 0.5)
RBK_SHIM_CONSTANT(one_div_root_two, 0.707106781186547524400844362104849039284835937688474036588)
RBK_SHIM_CONSTANT(root_two, 1.41421356237309504880168872420969807856967187537694807318)
RBK_SHIM_CONSTANT(half_root_two, 0.707106781186547524400844362104849039284835937688474036588)
RBK_SHIM_CONSTANT(pi, 3.14159265358979323846264338327950288419716939937510582097)
RBK_SHIM_CONSTANT(half_pi, 1.57079632679489661923132169163975144209858469968755291049)
RBK_SHIM_CONSTANT(two_pi, 6.28318530717958647692528676655900576839433879875021164195)

#undef RBK_SHIM_CONSTANT

}}} // namespace boost::math::constants

#endif
