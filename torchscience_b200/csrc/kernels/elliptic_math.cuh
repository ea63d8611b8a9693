// Complete elliptic integrals K(m), E(m) (parameter convention) and their
// first and second derivatives in m.
//
// The reference evaluates K = R_F(0, 1-m, 1) and E = 2 R_G(0, 1-m, 1) by
// Carlson duplication (complete_legendre_elliptic_integral_k.h:29-33,
// complete_legendre_elliptic_integral_e.h:71-79) and differentiates E by a
// central difference with h = 1e-6 (complete_legendre_elliptic_integral_e_backward.h:41-52).
// Here both come from one arithmetic-geometric mean sweep (DLMF 19.8.1 and
// 19.8.6): a_{n+1} = (a+b)/2, b_{n+1} = sqrt(ab), c_{n+1} = (a-b)/2 from
// a_0 = 1, b_0 = sqrt(1-m); K = π/(2 a_N), E = K (1 - Σ 2^(n-1) c_n²) with
// c_0² = m.  The sweep converges quadratically (≈ 7 steps at m = 1 - 1e-9).
// For m > 0.9 the values come instead from the complementary-parameter
// expansions in m1 = 1 - m (DLMF 19.12.1, 19.12.2), which carry the
// logarithmic singularity explicitly and avoid E = K(1 - Σ) cancelling by a
// factor ~K near m = 1.
// Derivatives use the closed forms (DLMF 19.4.1)
//   dK/dm = (E - (1-m)K) / (2m(1-m)),  dE/dm = (E - K) / (2m)
// and their m-derivatives; for small |m| these cancel, so there the
// Maclaurin series K = π/2 Σ c_n m^n, c_n = ((2n-1)!!/(2n)!!)² (DLMF 19.5.1)
// and its E counterpart are summed instead.
#pragma once

#include <math_constants.h>

namespace tsb {

template <typename T>
struct EllipKE {
  T K, E;      // values
  T Kp, Ep;    // d/dm
  T Kpp, Epp;  // d²/dm²
};

template <typename T>
__device__ __forceinline__ T sqrt_t(T v);
template <>
__device__ __forceinline__ double sqrt_t<double>(double v) { return sqrt(v); }
template <>
__device__ __forceinline__ float sqrt_t<float>(float v) { return sqrtf(v); }

// Maclaurin series for |m| small: K, E and derivatives up to ORDER.
template <typename T, int ORDER, int NTERMS>
__device__ inline EllipKE<T> ellip_series(T m) {
  EllipKE<T> r;
  T c = 1;        // c_n
  T mp = 1;       // m^n
  T mp1 = 0;      // m^(n-1)   (n >= 1)
  T mp2 = 0;      // m^(n-2)   (n >= 2)
  T K = 1, E = 1, Kp = 0, Ep = 0, Kpp = 0, Epp = 0;
#pragma unroll
  for (int n = 1; n <= NTERMS; ++n) {
    const T f = T(2 * n - 1) / T(2 * n);
    c *= f * f;
    mp2 = mp1;
    mp1 = mp;
    mp *= m;
    const T inv = T(1) / T(2 * n - 1);
    K += c * mp;
    E -= c * mp * inv;
    if (ORDER >= 1) {
      Kp += T(n) * c * mp1;
      Ep -= T(n) * c * mp1 * inv;
    }
    if (ORDER >= 2 && n >= 2) {
      Kpp += T(n * (n - 1)) * c * mp2;
      Epp -= T(n * (n - 1)) * c * mp2 * inv;
    }
  }
  const T h = T(CUDART_PIO2);
  r.K = h * K;
  r.E = h * E;
  r.Kp = h * Kp;
  r.Ep = h * Ep;
  r.Kpp = h * Kpp;
  r.Epp = h * Epp;
  return r;
}

template <typename T>
__device__ __forceinline__ T log_t(T v);
template <>
__device__ __forceinline__ double log_t<double>(double v) { return log(v); }
template <>
__device__ __forceinline__ float log_t<float>(float v) { return logf(v); }

// K(m), E(m) for m1 = 1 - m small (m1 < 0.1):
//   K = Σ c_n m1^n (L + d_n),  E = 1 + (m1/2) Σ e_n m1^n (L + d_n - 1/((2n+1)(2n+2)))
// with L = -ln(m1)/2, c_n = ((1/2)_n/n!)², e_n = (1/2)_n (3/2)_n / ((2)_n n!),
// d_0 = ln 4, d_n = d_{n-1} - 2/((2n-1)(2n)).
template <typename T, int NTERMS>
__device__ inline void ellip_comp_series(T m1, T& K, T& E) {
  const T L = T(-0.5) * log_t<T>(m1);
  T c = 1, ce = 1, d = T(1.3862943611198906), p = 1, k = 0, e = 0;
#pragma unroll
  for (int n = 0; n < NTERMS; ++n) {
    k += c * p * (L + d);
    e += ce * p * (L + d - T(1) / T((2 * n + 1) * (2 * n + 2)));
    c *= (T(2 * n + 1) / T(2 * n + 2)) * (T(2 * n + 1) / T(2 * n + 2));
    ce *= T((2 * n + 1) * (2 * n + 3)) / T(4 * (n + 2) * (n + 1));
    d -= T(2) / T((2 * n + 1) * (2 * n + 2));
    p *= m1;
  }
  K = k;
  E = T(1) + T(0.5) * m1 * e;
}

template <typename T, int ORDER>
__device__ inline EllipKE<T> ellip_agm(T m) {
  EllipKE<T> r;
  // Stop once c_{n+1} <= tol·a_{n+1} with tol ~ sqrt(eps): convergence is
  // quadratic, so the next c would be ~tol²/4·a, below the working precision,
  // and a_{n+1} already equals the mean to within it.  (A test against eps
  // itself can stall with a, b one ulp apart.)
  const T tol = sizeof(T) == 8 ? T(1e-8) : T(2.4e-4);
  T a = 1, b = sqrt_t<T>(T(1) - m);
  T sum = T(0.5) * m;  // 2^(n-1) c_n², n = 0
  T pw = T(0.5);
  for (int it = 0; it < (m > T(0.9) ? 0 : 40); ++it) {
    const T c = T(0.5) * (a - b);
    const T an = T(0.5) * (a + b);
    b = sqrt_t<T>(a * b);
    a = an;
    pw *= T(2);
    sum += pw * c * c;
    if (fabs(c) <= tol * a) break;
  }
  if (m > T(0.9)) {
    ellip_comp_series<T, sizeof(T) == 8 ? 17 : 8>(T(1) - m, r.K, r.E);
  } else {
    r.K = T(CUDART_PIO2) / a;
    r.E = r.K * (T(1) - sum);
  }
  r.Kp = r.Ep = r.Kpp = r.Epp = 0;
  if (ORDER >= 1) {
    const T mc = T(1) - m;
    r.Kp = (r.E - mc * r.K) / (T(2) * m * mc);
    r.Ep = (r.E - r.K) / (T(2) * m);
    if (ORDER >= 2) {
      const T N = r.E - mc * r.K, Dn = T(2) * m * mc;
      const T Np = r.Ep + r.K - mc * r.Kp, Dnp = T(2) * (T(1) - T(2) * m);
      r.Kpp = (Np * Dn - N * Dnp) / (Dn * Dn);
      r.Epp = (r.Ep - r.Kp) / (T(2) * m) - r.Ep / m;
    }
  }
  return r;
}

// K, E (+ derivatives) with the reference's domain conventions:
// NaN for m > 1 (sqrt of a negative in R_F), K(1) = +inf, E(1) = 1.
template <typename T, int ORDER>
__device__ inline EllipKE<T> ellip_eval(T m) {
  EllipKE<T> r;
  const T nan = T(CUDART_NAN), inf = T(CUDART_INF);
  if (isnan(m) || m > T(1)) {
    r.K = r.E = r.Kp = r.Ep = r.Kpp = r.Epp = nan;
    return r;
  }
  if (m == T(1)) {
    r.K = inf;
    r.E = T(1);
    r.Kp = inf;
    r.Ep = -inf;
    r.Kpp = inf;
    r.Epp = -inf;
    return r;
  }
  if (isinf(m)) {  // m = -inf
    r.K = T(0);
    r.E = inf;
    r.Kp = T(0);
    r.Ep = T(0);
    r.Kpp = T(0);
    r.Epp = T(0);
    return r;
  }
  // Below `small` the closed-form derivatives cancel by a factor ~1/m; the
  // Maclaurin series is used instead (FP32 needs the wider band).
  const T small = sizeof(T) == 8 ? T(0.1) : T(0.5);
  if (ORDER >= 1 && fabs(m) < small) return ellip_series<T, ORDER, sizeof(T) == 8 ? 20 : 26>(m);
  return ellip_agm<T, ORDER>(m);
}

template <int ORDER>
__device__ __forceinline__ EllipKE<double> ellip_t(double m) {
  return ellip_eval<double, ORDER>(m);
}
// Mixed kernels: the same algorithms entirely in FP32 (the complementary
// series removes the only cancellation that needed FP64).
template <int ORDER>
__device__ __forceinline__ EllipKE<float> ellip_t(float m) {
  return ellip_eval<float, ORDER>(m);
}

}  // namespace tsb
