// Beta-family evaluators in FP64: ln|B(a, b)|, B(a, b), the digamma and
// trigamma differences their derivatives need, and ψ^(n) of any order.
//
// Reference behaviour (kernel/special_functions/log_beta.h:10-13, beta.h:12-15,
// log_beta_backward.h:10-17, beta_backward.h:13-27, polygamma.h:12-62):
// ln B = lnΓ(a) + lnΓ(b) - lnΓ(a+b), B = exp(ln B), derivatives from
// ψ(a) - ψ(a+b), and ψ^(n) for n >= 4 from the recurrence to 6 and a
// three-term asymptotic series.  Those forms lose digits: lnΓ differences
// cancel when a or b is large (absolute error ε·lnΓ(a+b)), ψ(a) - ψ(a+b)
// cancels when b << a (relative error ε·ψ(a)/(b ψ'(a))), and the truncated
// series leaves a relative error of about 1e-6 at n = 4.  Here:
//
//   - ln B for a, b > 0: lnΓ sums while both are below 8; otherwise
//     Stirling's series (DLMF 5.11.1) with the logarithms combined so that
//     nothing large cancels:
//       ln B = (p - 1/2) ln(p/(p+q)) - (q - 1/2) log1p(p/q) - ln(p+q)/2
//              + ln(2π)/2 + μ(p) + μ(q) - μ(p+q)          (8 <= p <= q),
//       ln B = lnΓ(p) - (q - 1/2) log1p(p/q) - p ln(p+q) + p + μ(q) - μ(p+q)
//                                                        (p < 8 <= q),
//     μ the Stirling remainder Σ B_2k / (2k(2k-1) x^(2k-1)).
//   - ψ(x) - ψ(x+y) and ψ'(x) - ψ'(x+y) for x, y > 0: the recurrence terms
//     y/(x(x+y)) and y(2x+y)/(x²(x+y)²) (all of one sign) up to x >= 10, then
//     the difference of the asymptotic series term by term, each term a
//     difference of powers formed without cancellation.
//   - ψ^(n), n >= 4: (-1)^(n+1) n! ζ(n+1, z) with the Hurwitz zeta from
//     Euler–Maclaurin summation (direct terms up to Q >= 0.7(n+1) + 14,
//     then the integral, the half term and nine Bernoulli corrections), each
//     power scaled by n! directly, or in the logarithm where a power would
//     leave the normal range (so large orders neither overflow nor underflow
//     early); z < 0 by ζ(s, z) = ζ(s, z+m) + (-1)^s (ζ(s, f) -
//     ζ(s, f+m)), m = ⌈-z⌉, f = 1 - (z+m).
//
// Negative arguments: ln B keeps the reference's ln|B| from lnΓ sums; B is
// returned with its sign (the reference's exp(ln|B|) drops it).  A pole of
// Γ(a) or Γ(b) gives ln|B| = +inf and B = +inf (as the reference's tests
// expect at (0, 1) and (-1, 1)).
#pragma once

#include <math_constants.h>

#include "gamma_math.cuh"

namespace tsb {

namespace bt {
constexpr double kHalfLn2Pi = 0.91893853320467274;  // ln(2π)/2
constexpr double kSmall = 8.0;                       // Stirling's series for ln B from here on
constexpr double kPsi = 10.0;                        // asymptotic ψ, ψ' differences from here on
}  // namespace bt

// Stirling remainder μ(x) = lnΓ(x) - ((x - 1/2) ln x - x + ln(2π)/2), x >= 8.
__device__ __forceinline__ double stirling_mu(double x) {
  const double r = 1.0 / x, z = r * r;
  return r * (TSB_B2 / 2 + z * (TSB_B4 / 12 + z * (TSB_B6 / 30 + z * (TSB_B8 / 56 + z * (TSB_B10 / 90 +
             z * (TSB_B12 / 132 + z * (TSB_B14 / 182 + z * TSB_B16 / 240)))))));
}

// ln B(a, b) for a, b > 0.
__device__ inline double log_beta_pos(double a, double b) {
  const double p = fmin(a, b), q = fmax(a, b);
  if (q < bt::kSmall) return (lgamma(p) + lgamma(q)) - lgamma(p + q);
  const double s = p + q;
  const double lq = -(q - 0.5) * log1p(p / q) + (stirling_mu(q) - stirling_mu(s));
  if (p < bt::kSmall) return lgamma(p) + ((lq - p * log(s)) + p);
  return (((p - 0.5) * log(p / s) + lq) - 0.5 * log(s)) + (bt::kHalfLn2Pi + stirling_mu(p));
}

// ψ(x) - ψ(x + y) for x > 0, y > 0.
__device__ inline double psi_diff(double x, double y) {
  double acc = 0.0;
  while (x < bt::kPsi) {  // ψ(x) - ψ(x+y) = [ψ(x+1) - ψ(x+y+1)] - y/(x(x+y))
    acc -= y / (x * (x + y));
    x += 1.0;
  }
  // ψ(x) ~ ln x - 1/(2x) - Σ B_2k/(2k x^2k): difference term by term, with
  // D_k = x^-2k - X^-2k from D_{k+1} = D_k/x² + X^-2k (1/x² - 1/X²).
  const double X = x + y, rx = 1.0 / x, rX = 1.0 / X;
  const double rx2 = rx * rx, rX2 = rX * rX;
  const double d1 = y * (x + X) * rx2 * rX2;  // 1/x² - 1/X²
  const double bern[8] = {TSB_B2 / 2, TSB_B4 / 4, TSB_B6 / 6, TSB_B8 / 8, TSB_B10 / 10, TSB_B12 / 12, TSB_B14 / 14, TSB_B16 / 16};
  double D = d1, Xp = rX2, tail = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    tail = fma(bern[k], D, tail);
    D = fma(D, rx2, Xp * d1);
    Xp *= rX2;
  }
  return acc + ((-log1p(y * rx) - 0.5 * y * rx * rX) - tail);
}

// ψ'(x) - ψ'(x + y) for x > 0, y > 0.
__device__ inline double psi1_diff(double x, double y) {
  double acc = 0.0;
  while (x < bt::kPsi) {  // ψ'(x) = ψ'(x+1) + 1/x²
    const double X = x + y;
    acc += y * (x + X) / (x * x * X * X);
    x += 1.0;
  }
  // ψ'(x) ~ 1/x + 1/(2x²) + Σ B_2k / x^(2k+1): E_k = x^-(2k+1) - X^-(2k+1),
  // E_{k+1} = E_k/x² + X^-(2k+1) (1/x² - 1/X²).
  const double X = x + y, rx = 1.0 / x, rX = 1.0 / X;
  const double rx2 = rx * rx, rX2 = rX * rX;
  const double d1 = y * (x + X) * rx2 * rX2;  // 1/x² - 1/X²
  const double e1 = y * rx * rX;              // 1/x - 1/X
  const double bern[9] = {TSB_B2, TSB_B4, TSB_B6, TSB_B8, TSB_B10, TSB_B12, TSB_B14, TSB_B16, TSB_B18};
  double E = fma(e1, rx2, rX * d1), Xp = rX * rX2, tail = 0.0;  // E_1 = 1/x³ - 1/X³
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    tail = fma(bern[k], E, tail);
    E = fma(E, rx2, Xp * d1);
    Xp *= rX2;
  }
  return acc + ((e1 + 0.5 * d1) + tail);
}

__device__ __forceinline__ bool beta_pole(double v) { return v <= 0.0 && v == floor(v); }

// Sign of Γ(v) away from its poles.
__device__ __forceinline__ double gamma_sign(double v) {
  return v > 0.0 ? 1.0 : (fmod(ceil(-v), 2.0) == 1.0 ? -1.0 : 1.0);
}

// ln|B(a, b)|.
__device__ inline double log_beta_d(double a, double b) {
  if (isnan(a) || isnan(b)) return a + b;
  if (beta_pole(a) || beta_pole(b)) return CUDART_INF;
  if (a > 0.0 && b > 0.0) return isinf(a) || isinf(b) ? -CUDART_INF : log_beta_pos(a, b);
  return (lgamma_d(a) + lgamma_d(b)) - lgamma_d(a + b);
}

// B(a, b) with its sign.
__device__ inline double beta_d(double a, double b) {
  const double l = log_beta_d(a, b);
  if (!(a > 0.0 && b > 0.0) && isfinite(l)) return gamma_sign(a) * gamma_sign(b) * gamma_sign(a + b) * exp(l);
  return exp(l);
}

// ∂ ln B/∂a = ψ(a) - ψ(a+b), ∂ ln B/∂b = ψ(b) - ψ(a+b).
__device__ __forceinline__ double log_beta_da(double a, double b) {
  if (a > 0.0 && b > 0.0) return psi_diff(a, b);
  return digamma_d(a) - digamma_d(a + b);
}
// ∂² ln B/∂a² = ψ'(a) - ψ'(a+b).
__device__ __forceinline__ double log_beta_daa(double a, double b) {
  if (a > 0.0 && b > 0.0) return psi1_diff(a, b);
  return trigamma_d(a) - trigamma_d(a + b);
}

// ---------------------------------------------------------------- ψ^(n)
// n!·ζ(n+1, q) for q > 0.  Each power n!·v^-s is F·pow(v, -s) with F = n!
// in double (exact while n <= 22) when no v^-s of the call leaves the
// normal range, else exp(L - s ln v) with L = ln n!.
__device__ inline double hurwitz_scaled(int n, double L, double F, double q) {
  const double s = n + 1.0;
  const double qmin = fma(0.7, s, 14.0);
  const int N = q < qmin ? (int)ceil(qmin - q) : 0;
  const double Q = q + N;
  const double lQ = log(Q);
  const bool exact = n <= 170 && s * lQ < 700.0 && s * fabs(log(q)) < 700.0;
  const double base = exact ? F * pow(Q, -s) : exp(L - s * lQ);  // n!·Q^-s
  // Euler–Maclaurin tail: n!·[Q^(1-s)/(s-1) + Q^-s/2 + Σ_j B_2j/(2j)! (s)_(2j-1) Q^(-s-2j+1)]
  const double rQ = 1.0 / Q, rQ2 = rQ * rQ;
  const double bern[9] = {TSB_B2, TSB_B4, TSB_B6, TSB_B8, TSB_B10, TSB_B12, TSB_B14, TSB_B16, TSB_B18};
  double t = base * s * rQ / 2.0;  // j = 1 without B_2: n! s Q^(-s-1) / 2!
  double corr = 0.0;
#pragma unroll
  for (int j = 1; j <= 9; ++j) {
    corr = fma(bern[j - 1], t, corr);
    // (s)_(2j+1)/(2j+2)! = (s)_(2j-1)/(2j)! · (s+2j-1)(s+2j) / ((2j+1)(2j+2))
    t *= (s + 2 * j - 1) * (s + 2 * j) / ((2.0 * j + 1.0) * (2.0 * j + 2.0)) * rQ2;
  }
  double acc = (base * Q / n + 0.5 * base) + corr;
  for (int k = N - 1; k >= 0; --k) acc += exact ? F * pow(q + k, -s) : exp(L - s * log(q + k));
  return acc;
}

// ψ^(n)(z) for an integer order n >= 0.  n <= 3 use the dedicated
// evaluators; at the poles (z a non-positive integer) odd orders are +inf,
// even orders NaN (ψ itself -inf), as those evaluators give.
__device__ inline double polygamma_d(int n, double z) {
  if (n < 0 || isnan(z)) return CUDART_NAN;
  switch (n) {
    case 0: return digamma_d(z);
    case 1: return trigamma_d(z);
    case 2: return tetragamma_d(z);
    case 3: return pentagamma_d(z);
    default: break;
  }
  const bool odd = n & 1;
  if (isinf(z)) return z > 0.0 ? (odd ? 0.0 : -0.0) : CUDART_NAN;
  if (z <= 0.0 && z == floor(z)) return odd ? CUDART_INF : CUDART_NAN;
  const double L = lgamma((double)n + 1.0);
  double F = 1.0;  // n! (rounded above 22!; unused above 170)
  for (int i = 2; i <= min(n, 170); ++i) F *= i;
  const double sgn = odd ? 1.0 : -1.0;  // (-1)^(n+1)
  if (z > 0.0) return sgn * hurwitz_scaled(n, L, F, z);
  const double m = ceil(-z), zm = z + m, f = 1.0 - zm;
  return sgn * hurwitz_scaled(n, L, F, zm) + (hurwitz_scaled(n, L, F, f) - hurwitz_scaled(n, L, F, f + m));
}

// The order as the reference reads it: truncated toward zero
// (polygamma.h:47, static_cast<int>(n)); negative orders give NaN.
__device__ __forceinline__ int polygamma_order(double n) {
  if (isnan(n) || n <= -1.0) return -1;
  return n > 1e6 ? 1000000 : (int)n;
}

}  // namespace tsb
