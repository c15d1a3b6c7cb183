// Test infrastructure: a stand-in for the one Boost.Math function the
// reference's functionals call, so that alsfvm/src/functional/Legendre.cpp
// (lines 79-81) and LegendrePointWise.cpp (line 74) compile into the
// reference build here.  Boost is not in this image.
//
// boost::math::legendre_p(int l, T x) as Boost.Math documents it
// (special_functions/legendre.hpp; the reference's headers cite the
// Boost 1.46 documentation, and the function has kept this behaviour since),
// restated with the library's default policy:
//   * a double argument is evaluated in long double (policy promote_double),
//     and the result is rounded to double once at the end;
//   * |x| > 1 raises a domain error (std::domain_error under the default
//     throw_on_error policy);
//   * a negative degree l is evaluated as degree -l - 1 (P_{-l-1} = P_l);
//   * P_0 = 1, P_1 = x and Bonnet's recurrence
//     P_{n+1} = ((2n + 1) x P_n - n P_{n-1}) / (n + 1), its terms formed
//     left to right as written.
// Moment.cpp includes this header and calls nothing from it.
#pragma once

#include <stdexcept>
#include <string>

namespace boost {
namespace math {

namespace shim_detail {

inline long double legendre_eval(unsigned l, long double x) {
    if (x < -1 || x > 1) {
        throw std::domain_error("boost::math::legendre_p: the Legendre polynomial is defined for "
                                "-1 <= x <= 1, but got x = " + std::to_string(double(x)));
    }
    long double p0 = 1;
    long double p1 = x;
    if (l == 0) {
        return p0;
    }
    for (unsigned n = 1; n < l; ++n) {
        const long double next = ((2 * n + 1) * x * p1 - n * p0) / (n + 1);
        p0 = p1;
        p1 = next;
    }
    return p1;
}

} // namespace shim_detail

inline double legendre_p(int l, double x) {
    const unsigned degree = l < 0 ? unsigned(-l - 1) : unsigned(l);
    return double(shim_detail::legendre_eval(degree, static_cast<long double>(x)));
}

} // namespace math
} // namespace boost
