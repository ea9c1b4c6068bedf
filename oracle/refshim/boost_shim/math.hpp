// Stand-in for the three Boost.Math special functions the reference's initial
// conditions call (TEST INFRASTRUCTURE; Boost is not in this image):
//   boost::math::cyl_bessel_k(order, x)   initial_distributions.cpp:309, :355-357
//   boost::math::ellint_1(k, phi)          initial_distributions.cpp:419-420
//   boost::math::ellint_2(k, phi)
// Boost and the C++17 standard library use the same conventions here (K_nu(x);
// incomplete integrals of the first and second kind with modulus k and
// amplitude phi), so each maps to its std:: namesake.  Against Boost 1.78
// itself the values agree to rounding, not bit for bit.
#ifndef FS_ORACLE_BOOST_MATH_SHIM
#define FS_ORACLE_BOOST_MATH_SHIM

#include <cmath>

namespace boost {
namespace math {

template <typename T1, typename T2>
inline double cyl_bessel_k(T1 order, T2 x) {
    return std::cyl_bessel_k(static_cast<double>(order), static_cast<double>(x));
}

template <typename T1, typename T2>
inline double ellint_1(T1 k, T2 phi) {
    return std::ellint_1(static_cast<double>(k), static_cast<double>(phi));
}

template <typename T1, typename T2>
inline double ellint_2(T1 k, T2 phi) {
    return std::ellint_2(static_cast<double>(k), static_cast<double>(phi));
}

}  // namespace math
}  // namespace boost

#endif
