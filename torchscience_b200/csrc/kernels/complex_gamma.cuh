// The gamma family of complex argument (complex64 / complex128 data, both
// evaluated in complex128): lnΓ, Γ, ψ, ψ', ψ'', ψ'''.
//
// lnΓ is the principal branch ("loggamma"): analytic on C minus (-inf, 0],
// equal to ln Γ(x) on the positive reals, taken from above on the negative
// real axis (Im lnΓ(x + 0i) = -kπ with k the number of poles passed), and
// lnΓ(conj z) = conj lnΓ(z).  The reference's complex log_gamma
// (kernel/special_functions/log_gamma.h) is a sum of principal logarithms
// over Lanczos and reflection terms whose imaginary part can differ from
// this branch by a multiple of 2π; exp of the two agrees.
//
// Algorithms (published mathematics):
//   - Re z >= 10: Stirling's series (DLMF 5.11.1) to the z^-15 term; below,
//     the recurrence lnΓ(z) = lnΓ(z + n) - Σ Log(z + k) (each Log principal:
//     on C minus (-inf, 0] both sides are analytic and agree on the positive
//     reals, so the identity holds with principal logarithms);
//   - Re z < -8: the reflection Γ(z)Γ(1-z) = π / sin(πz) (DLMF 5.5.3) with
//     the branch fixed by lnΓ(z) = ln π - Log sin(πz) - lnΓ(1-z) + 2πi m,
//     m = -ceil(-1/4 - x/2) for Im z >= 0: the large-|y| limit of
//     Im[lnΓ(z) + lnΓ(1-z)] is (x - 1/2)π, and Log sin(πz) jumps only on
//     the lines x = -1/2 + 2j, where the imaginary part of sin(πz) is taken
//     as +0 here;
//   - ψ^(n): the same recurrence and asymptotic series (DLMF 5.15.8) and
//     the reflection formulas obtained by differentiating
//     ψ(z) = ψ(1-z) - π cot(πz) (DLMF 5.5.4).
#pragma once

#include <cuda/std/complex>
#include <math_constants.h>

namespace tsb {

using cdouble = cuda::std::complex<double>;

namespace cg {

constexpr double kHalfLn2Pi = 0.91893853320467274178;  // ½ ln 2π
constexpr double kLnPi = 1.14472988584940017414;       // ln π

__device__ __forceinline__ bool is_pole(cdouble z) {
  return z.imag() == 0.0 && z.real() <= 0.0 && z.real() == floor(z.real());
}

// sin(πz) and cos(πz) for |Im z| <= 20 (beyond, callers use the exponential
// limits); sinpi / cospi are exact at the integers and half-integers.
__device__ __forceinline__ void sincos_pi(cdouble z, cdouble& s, cdouble& c) {
  const double x = z.real(), y = z.imag();
  const double sx = sinpi(x), cx = cospi(x), ch = cosh(CUDART_PI * y), sh = sinh(CUDART_PI * y);
  s = cdouble(sx * ch, cx * sh);
  c = cdouble(cx * ch, -sx * sh);
}

// Stirling's series for lnΓ(w), Re w >= 10: (w - ½) Log w - w + ½ ln 2π +
// Σ_{k=1..8} B_2k / (2k (2k-1) w^(2k-1)); the next term is below 2e-18 |w|^-17.
__device__ inline cdouble lgamma_stirling(cdouble w) {
  const cdouble r = 1.0 / w, r2 = r * r;
  cdouble s = -3617.0 / 122400.0;
  s = s * r2 + 1.0 / 156.0;
  s = s * r2 - 691.0 / 360360.0;
  s = s * r2 + 1.0 / 1188.0;
  s = s * r2 - 1.0 / 1680.0;
  s = s * r2 + 1.0 / 1260.0;
  s = s * r2 - 1.0 / 360.0;
  s = s * r2 + 1.0 / 12.0;
  return (w - 0.5) * cuda::std::log(w) - w + double{kHalfLn2Pi} + s * r;
}

// lnΓ for Re z >= -8 (Im z of either sign): shift to Re >= 10.
__device__ inline cdouble lgamma_shifted(cdouble z) {
  const double x = z.real();
  if (x >= 10.0) return lgamma_stirling(z);
  const int n = (int)ceil(10.0 - x);
  double lnmod = 0.0, arg = 0.0;
  double prod = 1.0;  // Π |z+k|², folded into lnmod before it can overflow
  for (int k = 0; k < n; ++k) {
    const double re = x + k, im = z.imag();
    prod *= re * re + im * im;
    arg += atan2(im, re);
    if (prod > 1e280 || prod < 1e-280) {
      lnmod += 0.5 * log(prod);
      prod = 1.0;
    }
  }
  lnmod += 0.5 * log(prod);
  return lgamma_stirling(z + (double)n) - cdouble(lnmod, arg);
}

// Log sin(πz) for Im z >= 0 (see the header: on the lines x = -1/2 + 2j the
// imaginary part of sin(πz) is taken as +0).
__device__ inline cdouble log_sin_pi_upper(cdouble z) {
  const double x = z.real(), y = z.imag();
  double cx = cospi(x);
  if (cx == 0.0) cx = 0.0;  // +0
  const double sx = sinpi(x);
  if (y > 20.0) {
    // sin(πz) = (e^{πy}/2) (sin πx + i cos πx) (1 + O(e^{-2πy}))
    return cdouble(CUDART_PI * y - CUDART_LN2, atan2(cx, sx));
  }
  const double ch = cosh(CUDART_PI * y), sh = sinh(CUDART_PI * y);
  const double re = sx * ch, im = cx * sh;
  return cdouble(0.5 * log(sx * sx + sh * sh), atan2(im, re));
}

}  // namespace cg

__device__ inline cdouble loggamma_c(cdouble z) {
  double x = z.real(), y = z.imag();
  if (isnan(x) || isnan(y)) return cdouble(CUDART_NAN, CUDART_NAN);
  if (cg::is_pole(z)) return cdouble(CUDART_INF, 0.0);
  if (isinf(x) && x > 0.0 && isfinite(y)) return cdouble(CUDART_INF, 0.0);
  if (isinf(x) || isinf(y)) return cdouble(CUDART_NAN, CUDART_NAN);
  const bool lower = signbit(y);
  if (lower) y = -y;
  const cdouble w(x, y);
  cdouble r;
  if (x < -8.0) {
    const double m = -ceil(-0.25 - 0.5 * x);
    r = double{cg::kLnPi} - cg::log_sin_pi_upper(w) - cg::lgamma_shifted(1.0 - w) + cdouble(0.0, 2.0 * CUDART_PI * m);
  } else {
    r = cg::lgamma_shifted(w);
  }
  return lower ? cuda::std::conj(r) : r;
}

__device__ inline cdouble gamma_c(cdouble z) {
  if (cg::is_pole(z)) return cdouble(CUDART_INF, 0.0);
  return cuda::std::exp(loggamma_c(z));
}

namespace cg {

// ψ^(n)(w) asymptotic series for Re w >= 10 (n = 0..3), to the B_16 term.
template <int N>
__device__ inline cdouble polygamma_asym(cdouble w) {
  const cdouble r = 1.0 / w, r2 = r * r;
  // Bernoulli numbers B_2 .. B_16
  const double B[8] = {1.0 / 6, -1.0 / 30, 1.0 / 42, -1.0 / 30, 5.0 / 66, -691.0 / 2730, 7.0 / 6, -3617.0 / 510};
  if constexpr (N == 0) {
    // Log w - 1/(2w) - Σ B_2k / (2k w^2k)
    cdouble s = 0.0;
    for (int k = 7; k >= 0; --k) s = (s + B[k] / (2.0 * (k + 1))) * r2;
    return cuda::std::log(w) - 0.5 * r - s;
  } else if constexpr (N == 1) {
    // 1/w + 1/(2w²) + Σ B_2k / w^(2k+1)
    cdouble s = 0.0;
    for (int k = 7; k >= 0; --k) s = (s + B[k]) * r2;
    return r + 0.5 * r2 + s * r;
  } else if constexpr (N == 2) {
    // -1/w² - 1/w³ - Σ (2k+1) B_2k / w^(2k+2)
    cdouble s = 0.0;
    for (int k = 7; k >= 0; --k) s = (s + (2.0 * (k + 1) + 1.0) * B[k]) * r2;
    return -r2 - r2 * r - s * r2;
  } else {
    // 2/w³ + 3/w⁴ + Σ (2k+1)(2k+2) B_2k / w^(2k+3)
    cdouble s = 0.0;
    for (int k = 7; k >= 0; --k) s = (s + (2.0 * (k + 1) + 1.0) * (2.0 * (k + 1) + 2.0) * B[k]) * r2;
    return 2.0 * r2 * r + 3.0 * r2 * r2 + s * r2 * r;
  }
}

// ψ^(n)(z) for Re z >= -8: shift to Re >= 10 with
// ψ^(n)(z) = ψ^(n)(z + m) - (-1)^n n! Σ 1/(z+k)^(n+1).
template <int N>
__device__ inline cdouble polygamma_shifted(cdouble z) {
  const double x = z.real();
  const int m = x >= 10.0 ? 0 : (int)ceil(10.0 - x);
  cdouble acc = 0.0;
  for (int k = 0; k < m; ++k) {
    const cdouble q = 1.0 / (z + (double)k);
    cdouble t = q;
    for (int j = 0; j < N; ++j) t *= q;
    acc += t;
  }
  constexpr double sign_fact = N == 0 ? -1.0 : N == 1 ? 1.0 : N == 2 ? -2.0 : 6.0;  // -(-1)^n n!
  return polygamma_asym<N>(z + (double)m) + sign_fact * acc;
}

}  // namespace cg

// ψ^(n)(z), n = 0..3; NaN at the poles (the reference's complex reflection
// divides by sin(πz) = 0 there).
template <int N>
__device__ inline cdouble polygamma_c(cdouble z) {
  const double x = z.real(), y = z.imag();
  if (isnan(x) || isnan(y) || cg::is_pole(z) || isinf(x) || isinf(y)) return cdouble(CUDART_NAN, CUDART_NAN);
  if (x >= -8.0) return cg::polygamma_shifted<N>(z);
  // reflection: ψ(z) = ψ(1-z) - π cot(πz) and its derivatives
  //   ψ'(z)   = -ψ'(1-z) + π² / s²
  //   ψ''(z)  =  ψ''(1-z) - 2π³ c / s³
  //   ψ'''(z) = -ψ'''(1-z) + 2π⁴ (1/s⁴ + 2c²/s⁴)      (s = sin πz, c = cos πz)
  const cdouble other = cg::polygamma_shifted<N>(1.0 - z);
  const double pi = CUDART_PI;
  cdouble cot, csc2;  // cot(πz), 1/sin²(πz)
  if (fabs(y) > 20.0) {
    cot = cdouble(0.0, y > 0.0 ? -1.0 : 1.0);
    csc2 = 0.0;  // |1/sin²| ~ 4 e^{-2π|y|}
  } else {
    cdouble s, c;
    cg::sincos_pi(z, s, c);
    const cdouble rs = 1.0 / s;
    cot = c * rs;
    csc2 = rs * rs;
  }
  if constexpr (N == 0) return other - pi * cot;
  else if constexpr (N == 1) return -other + pi * pi * csc2;
  else if constexpr (N == 2) return other - 2.0 * pi * pi * pi * cot * csc2;
  else return -other + 2.0 * pi * pi * pi * pi * csc2 * (csc2 + 2.0 * cot * cot);
}

__device__ inline cdouble digamma_c(cdouble z) { return polygamma_c<0>(z); }
__device__ inline cdouble trigamma_c(cdouble z) { return polygamma_c<1>(z); }
__device__ inline cdouble tetragamma_c(cdouble z) { return polygamma_c<2>(z); }
__device__ inline cdouble pentagamma_c(cdouble z) { return polygamma_c<3>(z); }

}  // namespace tsb
