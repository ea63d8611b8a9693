// Bessel functions of real order: J_ν, Y_ν, I_ν, K_ν and their x-derivatives.
//
// The reference (bessel_j.h:240-316, bessel_y.h:131-193, modified_bessel_i.h:271-366,
// modified_bessel_k.h:249-307) uses ascending series up to x <= 20 + 2|ν| and
// a two-term Hankel expansion beyond, and connection formulas
// Y = (J cos νπ - J_-ν)/sin νπ, K = π/2 (I_-ν - I_ν)/sin νπ; these lose
// all accuracy for x > 20 (J, Y, I) and for 1 <= x < 60 (K).  This file
// evaluates the same functions by published methods chosen per region:
//
//   x < 2         J_ν, I_ν by the ascending series (DLMF 10.2.2, 10.25.2);
//                 Y_μ, Y_μ+1 and K_μ, K_μ+1 at the reduced order
//                 μ = ν - round(ν), |μ| <= 1/2, by Temme's series (Temme,
//                 J. Comput. Phys. 19 (1975)), then upward recurrence in the
//                 order (stable for Y and K);
//   2 <= x < 25   Steed's method: the continued fraction CF1 for
//   or ν >= x     J'_ν/J_ν (I'_ν/I_ν), downward recurrence to μ, the complex
//                 continued fraction CF2 at μ (Temme's variant for K), and
//                 normalisation by the Wronskian (Barnett et al., Comput.
//                 Phys. Commun. 8 (1974); Temme 1975);
//   x >= 25       Hankel's expansions at μ and μ+1 (DLMF 10.17.3, 10.40.1-2),
//                 then upward recurrence (stable for J, Y while ν < x; for I
//                 used while x >= ν²/2, where the error growth stays below e²).
//
// Negative orders use DLMF 10.4.6-7 (J, Y), 10.27.2-3 (I, K).  The Temme
// series needs g1(μ), g2(μ) (combinations of 1/Γ(1 ± μ)); they come from
// polynomial fits generated by fits/gen_fits.py.  All loops are capped.
#pragma once

#include "unconverged.cuh"
#include <math_constants.h>

#include "bessel01_math.cuh"
#include "fits.cuh"
#include "gamma_math.cuh"

namespace tsb {

namespace bx {
__device__ __forceinline__ double exp_(double v) { return exp(v); }
__device__ __forceinline__ float exp_(float v) { return expf(v); }
__device__ __forceinline__ double log_(double v) { return log(v); }
__device__ __forceinline__ float log_(float v) { return logf(v); }
__device__ __forceinline__ double sqrt_(double v) { return sqrt(v); }
__device__ __forceinline__ float sqrt_(float v) { return sqrtf(v); }
__device__ __forceinline__ double sin_(double v) { return sin(v); }
__device__ __forceinline__ float sin_(float v) { return sinf(v); }
__device__ __forceinline__ double sinh_(double v) { return sinh(v); }
__device__ __forceinline__ float sinh_(float v) { return sinhf(v); }
__device__ __forceinline__ double cosh_(double v) { return cosh(v); }
__device__ __forceinline__ float cosh_(float v) { return coshf(v); }
__device__ __forceinline__ double lgamma_(double v) { return lgamma(v); }
__device__ __forceinline__ float lgamma_(float v) { return lgammaf(v); }
__device__ __forceinline__ void sincos_(double v, double* s, double* c) { sincos(v, s, c); }
__device__ __forceinline__ void sincos_(float v, float* s, float* c) { sincosf(v, s, c); }
__device__ __forceinline__ void sincospi_(double v, double* s, double* c) { sincospi(v, s, c); }
__device__ __forceinline__ void sincospi_(float v, float* s, float* c) { sincospif(v, s, c); }
}  // namespace bx

template <typename T>
struct BesselK;
template <>
struct BesselK<double> {
  static constexpr double EPS = 1.1e-16;
  // Convergence of a continued fraction judged by its factor's distance
  // from 1: just over one unit of 1's spacing (2^-52), so that a factor that
  // settles one ulp above or below 1 ends the loop instead of running to
  // MAXIT (EPS alone accepts only a factor of exactly 1 or 1 - 2^-53).
  static constexpr double EPS_RATIO = 2.3e-16;
  static constexpr double FPMIN = 1e-300;
  static constexpr double BIG = 1e280;
  static constexpr int MAXIT = 20000;
};
template <>
struct BesselK<float> {
  static constexpr float EPS = 6e-8f;
  static constexpr float EPS_RATIO = 1.3e-7f;  // just over one unit of 1's spacing (2^-23), as above
  static constexpr float FPMIN = 1e-35f;
  static constexpr float BIG = 1e35f;
  static constexpr int MAXIT = 20000;
};

// Values and x-derivatives.  For I and K the "scaled" results of the x >= 2
// paths carry e^{-x} I and e^{x} K; bessel_ik() removes the scaling.
template <typename T>
struct JY {
  T j, jp, y, yp;
};
template <typename T>
struct IK {
  T i, ip, k, kp;
};

__device__ __forceinline__ void temme_gammas(double mu, double& g1, double& g2, double& gpl, double& gmi) {
  const double u = 2.0 * mu;
  g1 = horner(fits::TEMME_G1_D, u);
  g2 = horner(fits::TEMME_G2_D, u);
  gpl = g2 - mu * g1;  // 1/Γ(1+μ)
  gmi = g2 + mu * g1;  // 1/Γ(1-μ)
}
__device__ __forceinline__ void temme_gammas(float mu, float& g1, float& g2, float& gpl, float& gmi) {
  const float u = 2.0f * mu;
  g1 = horner(fits::TEMME_G1_F, u);
  g2 = horner(fits::TEMME_G2_F, u);
  gpl = g2 - mu * g1;
  gmi = g2 + mu * g1;
}

// Compensated (Kahan) accumulator: in FP32 the Temme sums below add ~20
// terms of one sign, whose plain rounding error exceeds 1e-6.
template <typename T>
struct Kahan {
  T s, c;
  __device__ __forceinline__ explicit Kahan(T v) : s(v), c(0) {}
  __device__ __forceinline__ void add(T v) {
    const T y = v - c;
    const T t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

// Ascending series of J_ν (sgn = -1) or I_ν (sgn = +1) and its x-derivative:
// C_ν = (x/2)^ν/Γ(ν+1) Σ t_k, t_k = t_{k-1} (sgn x²/4) / (k (ν+k)),
// C'_ν = (x/2)^ν/Γ(ν+1) Σ t_k (ν + 2k) / x.
template <typename T>
__device__ inline void bessel_series(T nu, T x, T sgn, T& val, T& der) {
  const T eps = BesselK<T>::EPS;
  const T h = T(0.5) * x, q = sgn * h * h;
  T t = 1, s = 1, sd = nu;
  {  // counted loop: reaching the cap is recorded (note_unconverged)
    int k = 1;
    for (; k < 500; ++k) {
      t *= q / (T(k) * (nu + T(k)));
      s += t;
      const T td = t * (nu + T(2 * k));
      sd += td;
      if (fabs(t) <= eps * fabs(s) && fabs(td) <= eps * fabs(sd)) break;
    }
    if (k >= 500) note_unconverged();
  }
  // (x/2)^ν / Γ(ν+1): its exponent reaches a few hundred, so in the FP32
  // kernels it is formed in FP64 (an FP32 exponent would cost ~1e-5).
  // The products are formed in FP64 too: the prefactor alone can be an FP32
  // denormal while the value is not.
  const double pre = exp((double)nu * log((double)h) - lgamma((double)nu + 1.0));
  val = (T)(pre * (double)s);
  der = (T)(pre * (double)sd / (double)x);
}

// Temme's series for Y_μ, Y_{μ+1} (|μ| <= 1/2, 0 < x < 2).
template <typename T>
__device__ inline void temme_y(T mu, T x, T& ymu, T& ymu1) {
  const T eps = BesselK<T>::EPS, pi = T(CUDART_PI);
  const T x2 = T(0.5) * x, pimu = pi * mu;
  const T fact = fabs(pimu) < eps ? T(1) : pimu / bx::sin_(pimu);
  const T d = -bx::log_(x2), e = mu * d;
  const T fact2 = fabs(e) < eps ? T(1) : bx::sinh_(e) / e;
  T g1, g2, gpl, gmi;
  temme_gammas(mu, g1, g2, gpl, gmi);
  T ff = T(2) / pi * fact * (g1 * bx::cosh_(e) + g2 * fact2 * d);
  const T ee = bx::exp_(e);
  T p = ee / (gpl * pi);
  T q = T(1) / (ee * pi * gmi);
  const T pimu2 = T(0.5) * pimu;
  const T fact3 = fabs(pimu2) < eps ? T(1) : bx::sin_(pimu2) / pimu2;
  const T r = pi * pimu2 * fact3 * fact3;
  T c = 1;
  Kahan<T> sum(ff + r * q), sum1(p);
  const T dd = -x2 * x2;
  {  // counted loop: reaching the cap is recorded (note_unconverged)
    int i = 1;
    for (; i < 500; ++i) {
      const T fi = T(i);
      ff = (fi * ff + p + q) / (fi * fi - mu * mu);
      c *= dd / fi;
      p /= (fi - mu);
      q /= (fi + mu);
      const T del = c * (ff + r * q);
      sum.add(del);
      const T del1 = c * p - fi * del;
      sum1.add(del1);
      if (fabs(del) < (T(1) + fabs(sum.s)) * eps && fabs(del1) < (T(1) + fabs(sum1.s)) * eps) break;
    }
    if (i >= 500) note_unconverged();
  }
  ymu = -sum.s;
  ymu1 = -sum1.s * (T(2) / x);
}

// Temme's series for K_μ, K_{μ+1} (|μ| <= 1/2, 0 < x < 2), unscaled.
template <typename T>
__device__ inline void temme_k(T mu, T x, T& kmu, T& kmu1) {
  const T eps = BesselK<T>::EPS, pi = T(CUDART_PI);
  const T x2 = T(0.5) * x, pimu = pi * mu;
  const T fact = fabs(pimu) < eps ? T(1) : pimu / bx::sin_(pimu);
  const T d = -bx::log_(x2), e = mu * d;
  const T fact2 = fabs(e) < eps ? T(1) : bx::sinh_(e) / e;
  T g1, g2, gpl, gmi;
  temme_gammas(mu, g1, g2, gpl, gmi);
  T ff = fact * (g1 * bx::cosh_(e) + g2 * fact2 * d);
  Kahan<T> sum(ff);
  const T ee = bx::exp_(e);
  T p = T(0.5) * ee / gpl;
  T q = T(0.5) / (ee * gmi);
  T c = 1;
  Kahan<T> sum1(p);
  const T dd = x2 * x2;
  {  // counted loop: reaching the cap is recorded (note_unconverged)
    int i = 1;
    for (; i < 500; ++i) {
      const T fi = T(i);
      ff = (fi * ff + p + q) / (fi * fi - mu * mu);
      c *= dd / fi;
      p /= (fi - mu);
      q /= (fi + mu);
      const T del = c * ff;
      sum.add(del);
      const T del1 = c * (p - fi * ff);
      sum1.add(del1);
      if (fabs(del) < fabs(sum.s) * eps && fabs(del1) < fabs(sum1.s) * eps) break;
    }
    if (i >= 500) note_unconverged();
  }
  kmu = sum.s;
  kmu1 = sum1.s * (T(2) / x);
}

// Upward recurrence C_{k+1} = (2k/x) C_k - s C_{k-1} from order mu to mu + n
// (s = 1: J, Y; s = -1: K).  On return c0 = C_{mu+n}, c1 = C_{mu+n+1}.  A
// value that overflows becomes an infinity of its sign (C_{mu+n+1} may
// overflow while C_{mu+n} does not).
template <typename T>
__device__ inline void recur_up(T mu, T x, int n, T s, T& c0, T& c1) {
  const T xi2 = T(2) / x;
  for (int i = 1; i <= n; ++i) {
    const T t = (mu + T(i)) * xi2 * c1 - s * c0;
    if (isinf(t) || isnan(t)) {
      const T sinf = copysign(T(CUDART_INF), c1);
      if (i < n) {
        c0 = sinf;
        c1 = sinf;
      } else {
        c0 = c1;
        c1 = sinf;
      }
      return;
    }
    c0 = c1;
    c1 = t;
  }
}

// recur_up with the recurrence carried in FP64 for both flavours (for
// double data it is recur_up itself): a few FP64 operations per step with no
// division, where FP32 would add ~1e-6 over ~20 steps.
template <typename T>
__device__ __forceinline__ void recur_up_fp64(T mu, T x, int n, T s, T& c0, T& c1) {
  double d0 = c0, d1 = c1;
  recur_up<double>((double)mu, (double)x, n, (double)s, d0, d1);
  c0 = (T)d0;
  c1 = (T)d1;
}

// Hankel's asymptotic sums for x >= 25 (DLMF 10.17.3, 10.40.1-2):
//   P = Σ (-1)^k a_2k / x^2k,  Q = Σ (-1)^k a_2k+1 / x^2k+1,  S± = Σ (±1)^k a_k / x^k,
// a_k(ν) = Π_{j<=k} (4ν² - (2j-1)²) / (k! 8^k).  Stops at convergence or when
// the asymptotic terms start to grow.
template <typename T>
__device__ inline void hankel_sums(T nu, T x, T& P, T& Q, T& Sp, T& Sm) {
  const T eps = BesselK<T>::EPS;
  const T m = T(4) * nu * nu, z = T(1) / (T(8) * x);
  T term = 1, prev = T(CUDART_INF);
  P = 1;
  Q = 0;
  Sp = 1;
  Sm = 1;
  for (int k = 1; k < 60; ++k) {
    const T odd = T(2 * k - 1);
    term *= (m - odd * odd) * z / T(k);
    const T at = fabs(term);
    if (at > prev) break;
    prev = at;
    const int r = k & 3;  // k mod 4 selects the sign in P, Q
    if (k & 1) Q += (r == 1) ? term : -term;
    else P += (r == 0) ? term : -term;
    Sp += term;
    Sm += (k & 1) ? -term : term;
    if (at <= eps * (fabs(P) + fabs(Q))) break;
  }
}

// J_ν, J'_ν, Y_ν, Y'_ν for ν >= 0, 0 < x < inf.  NEED_J false: only Y
// (the series and Hankel regions then skip J's sum and recurrence; Steed's
// method yields both together).
template <typename T, bool NEED_Y, bool NEED_J = true>
__device__ inline JY<T> besseljy_pos(T nu, T x) {
  const T eps = BesselK<T>::EPS, fpmin = BesselK<T>::FPMIN, pi = T(CUDART_PI);
  JY<T> r;
  r.j = r.jp = r.y = r.yp = T(0);
  if (x < T(2)) {
    if (NEED_J) bessel_series<T>(nu, x, T(-1), r.j, r.jp);
    if (NEED_Y) {
      const int nl = (int)(nu + T(0.5));
      const T mu = nu - T(nl);
      // Temme's series and the order recurrence in FP64 (both flavours): in
      // FP32 the series' second sum cancels and 20 recurrence steps add
      // ~1.5e-6.
      double y0, y1;
      temme_y<double>((double)mu, (double)x, y0, y1);
      recur_up<double>((double)mu, (double)x, nl, 1.0, y0, y1);
      r.y = (T)y0;
      r.yp = isinf(y0) ? T(CUDART_INF) : (T)((double)nu / (double)x * y0 - y1);
    }
    return r;
  }
  if (x >= T(25) && nu < x) {
    // Hankel at μ and μ + 1, then upward recurrence for J and Y.
    const int nl = (int)(nu + T(0.5));
    const T mu = nu - T(nl);
    T sx, cx;
    bx::sincos_(x, &sx, &cx);
    const T amp = bx::sqrt_(T(2) / (pi * x));
    T c[2][2];  // [order][J, Y]
#pragma unroll
    for (int o = 0; o < 2; ++o) {
      const T v = mu + T(o);
      T P, Q, Sp, Sm;
      hankel_sums<T>(v, x, P, Q, Sp, Sm);
      T sf, cf;
      bx::sincospi_(T(0.5) * v + T(0.25), &sf, &cf);
      const T cw = cx * cf + sx * sf;  // cos(x - φ)
      const T sw = sx * cf - cx * sf;  // sin(x - φ)
      c[o][0] = amp * (P * cw - Q * sw);
      c[o][1] = amp * (P * sw + Q * cw);
    }
    T j0 = c[0][0], j1 = c[1][0], y0 = c[0][1], y1 = c[1][1];
    if (NEED_J) {
      recur_up_fp64<T>(mu, x, nl, T(1), j0, j1);
      r.j = j0;
      r.jp = nu / x * j0 - j1;
    }
    if (NEED_Y) {
      recur_up_fp64<T>(mu, x, nl, T(1), y0, y1);
      r.y = y0;
      r.yp = nu / x * y0 - y1;
    }
    return r;
  }
  // Steed's method.
  const int nl = max(0, (int)(nu - x + T(1.5)));
  const T mu = nu - T(nl);
  const T xi = T(1) / x, xi2 = T(2) * xi, w = xi2 / pi;
  int isign = 1;
  T h = nu * xi;
  if (h < fpmin) h = fpmin;
  T b = xi2 * nu, d = 0, c = h;
  {  // counted loop: reaching the cap is recorded (note_unconverged)
    int i = 1;
    for (; i < BesselK<T>::MAXIT; ++i) {
      b += xi2;
      d = b - d;
      if (fabs(d) < fpmin) d = fpmin;
      c = b - T(1) / c;
      if (fabs(c) < fpmin) c = fpmin;
      d = T(1) / d;
      const T del = c * d;
      h *= del;
      if (d < T(0)) isign = -isign;
      if (fabs(del - T(1)) < BesselK<T>::EPS_RATIO) break;
    }
    if (i >= BesselK<T>::MAXIT) note_unconverged();
  }
  T rjl = T(isign) * fpmin, rjpl = h * rjl;
  T rjl1 = rjl, rjp1 = rjpl, fact = nu * xi;
  for (int l = nl; l >= 1; --l) {
    const T t = fact * rjl + rjpl;
    fact -= xi;
    rjpl = fact * t - rjl;
    rjl = t;
    if (fabs(rjl) > BesselK<T>::BIG) {  // rescale (the ratio is what matters)
      const T s = T(1) / BesselK<T>::BIG;
      rjl *= s;
      rjpl *= s;
      rjl1 *= s;
      rjp1 *= s;
    }
  }
  if (rjl == T(0)) rjl = eps;
  const T f = rjpl / rjl;
  // CF2: p + iq = (J'_μ + iY'_μ) / (J_μ + iY_μ)
  T a = T(0.25) - mu * mu, p = T(-0.5) * xi, q = 1;
  const T br = T(2) * x;
  T bi = 2;
  T fct = a * xi / (p * p + q * q);
  T cr = br + q * fct, ci = bi + p * fct;
  T den = br * br + bi * bi;
  T dr = br / den, di = -bi / den;
  T dlr = cr * dr - ci * di, dli = cr * di + ci * dr;
  T tmp = p * dlr - q * dli;
  q = p * dli + q * dlr;
  p = tmp;
  {  // counted loop: reaching the cap is recorded (note_unconverged)
    int i = 2;
    for (; i < BesselK<T>::MAXIT; ++i) {
      a += T(2 * (i - 1));
      bi += T(2);
      dr = a * dr + br;
      di = a * di + bi;
      if (fabs(dr) + fabs(di) < fpmin) dr = fpmin;
      fct = a / (cr * cr + ci * ci);
      cr = br + cr * fct;
      ci = bi - ci * fct;
      if (fabs(cr) + fabs(ci) < fpmin) cr = fpmin;
      den = dr * dr + di * di;
      dr /= den;
      di /= -den;
      dlr = cr * dr - ci * di;
      dli = cr * di + ci * dr;
      tmp = p * dlr - q * dli;
      q = p * dli + q * dlr;
      p = tmp;
      if (fabs(dlr - T(1)) + fabs(dli) < BesselK<T>::EPS_RATIO) break;
    }
    if (i >= BesselK<T>::MAXIT) note_unconverged();
  }
  const T gam = (p - f) / q;
  T rjmu = bx::sqrt_(w / ((p - f) * gam + q));
  rjmu = copysign(rjmu, rjl);
  const T rymu = rjmu * gam;
  const T rymup = rymu * (p + q / gam);
  const T ry1 = mu * xi * rymu - rymup;
  fact = rjmu / rjl;
  r.j = rjl1 * fact;
  r.jp = rjp1 * fact;
  if (NEED_Y) {
    T y0 = rymu, y1 = ry1;
    recur_up_fp64<T>(mu, x, nl, T(1), y0, y1);
    r.y = y0;
    r.yp = nu * xi * y0 - y1;
  }
  return r;
}

// I_ν, I'_ν, K_ν, K'_ν for ν >= 0, 0 < x < inf; for x >= 2 the results are
// scaled (e^{-x} I, e^{x} K) and `scaled` is set.
template <typename T, bool NEED_I, bool NEED_K>
__device__ inline IK<T> besselik_pos(T nu, T x, bool& scaled) {
  const T eps = BesselK<T>::EPS, fpmin = BesselK<T>::FPMIN, pi = T(CUDART_PI);
  IK<T> r;
  r.i = r.ip = r.k = r.kp = T(0);
  const int nl = (int)(nu + T(0.5));
  const T mu = nu - T(nl);
  if (x < T(2)) {
    scaled = false;
    if (NEED_I) bessel_series<T>(nu, x, T(1), r.i, r.ip);
    if (NEED_K) {
      double k0, k1;  // FP64 for both flavours, as for Y above
      temme_k<double>((double)mu, (double)x, k0, k1);
      recur_up<double>((double)mu, (double)x, nl, -1.0, k0, k1);
      r.k = (T)k0;
      r.kp = isinf(k0) ? -T(CUDART_INF) : (T)((double)nu / (double)x * k0 - k1);
    }
    return r;
  }
  scaled = true;
  const T xi = T(1) / x, xi2 = T(2) * xi;
  const bool large = x >= T(25);
  // K̃_μ, K̃_{μ+1} (scaled by e^x)
  T k0, k1;
  if (large) {
    T P, Q, Sp, Sm, P1, Q1, Sp1, Sm1;
    hankel_sums<T>(mu, x, P, Q, Sp, Sm);
    hankel_sums<T>(mu + T(1), x, P1, Q1, Sp1, Sm1);
    const T ak = bx::sqrt_(pi / (T(2) * x));
    k0 = ak * Sp;
    k1 = ak * Sp1;
  } else {
    // Temme's CF2 for K̃_μ (Steed's method for K).
    T b = T(2) * (T(1) + x), d = T(1) / b, h = d, delh = d;
    T q1 = 0, q2 = 1;
    const T a1 = T(0.25) - mu * mu;
    T q = a1, c = a1, a = -a1, s = T(1) + q * delh;
    {  // counted loop: reaching the cap is recorded (note_unconverged)
      int i = 2;
      for (; i < BesselK<T>::MAXIT; ++i) {
        a -= T(2 * (i - 1));
        c = -a * c / T(i);
        const T qn = (q1 - b * q2) / a;
        q1 = q2;
        q2 = qn;
        q += c * qn;
        b += T(2);
        d = T(1) / (b + a * d);
        delh = (b * d - T(1)) * delh;
        h += delh;
        const T dels = q * delh;
        s += dels;
        if (fabs(dels / s) < eps) break;
      }
      if (i >= BesselK<T>::MAXIT) note_unconverged();
    }
    h = a1 * h;
    k0 = bx::sqrt_(pi / (T(2) * x)) / s;
    k1 = k0 * (mu + x + T(0.5) - h) * xi;
  }
  if (NEED_I) {
    if (large && x >= T(0.5) * nu * nu) {
      T P, Q, Sp, Sm, P1, Q1, Sp1, Sm1;
      hankel_sums<T>(mu, x, P, Q, Sp, Sm);
      hankel_sums<T>(mu + T(1), x, P1, Q1, Sp1, Sm1);
      const T ai = T(1) / bx::sqrt_(T(2) * pi * x);
      T i0 = ai * Sm, i1 = ai * Sm1;
      // I_{k+1} = I_{k-1} - (2k/x) I_k; for x >= ν²/2 the error growth of
      // this (mildly unstable) upward recurrence stays below e².
      // the recurrence in FP64 for both flavours: a few FP64 operations per
      // step, where FP32 would add ~1e-6 over ~20 steps
      double d0 = i0, d1 = i1;
      const double dxi2 = (double)xi2;
      for (int i = 1; i <= nl; ++i) {
        const double t = d0 - ((double)mu + (double)i) * dxi2 * d1;
        d0 = d1;
        d1 = t;
      }
      r.i = (T)d0;
      r.ip = (T)((double)(nu * xi) * d0 + d1);
    } else {
      // CF1 for f = I'_ν/I_ν, downward recurrence to μ, Wronskian with K̃.
      T h = nu * xi;
      if (h < fpmin) h = fpmin;
      T b = xi2 * nu, d = 0, c = h;
      {  // counted loop: reaching the cap is recorded (note_unconverged)
        int i = 1;
        for (; i < BesselK<T>::MAXIT; ++i) {
          b += xi2;
          d = T(1) / (b + d);
          c = b + T(1) / c;
          const T del = c * d;
          h *= del;
          if (fabs(del - T(1)) < BesselK<T>::EPS_RATIO) break;
        }
        if (i >= BesselK<T>::MAXIT) note_unconverged();
      }
      T ril = fpmin, ripl = h * ril;
      T ril1 = ril, rip1 = ripl, fact = nu * xi;
      for (int l = nl; l >= 1; --l) {
        const T t = fact * ril + ripl;
        fact -= xi;
        ripl = fact * t + ril;
        ril = t;
        if (fabs(ril) > BesselK<T>::BIG) {
          const T s = T(1) / BesselK<T>::BIG;
          ril *= s;
          ripl *= s;
          ril1 *= s;
          rip1 *= s;
        }
      }
      const T f = ripl / ril;
      const T kmup = mu * xi * k0 - k1;
      const T rimu = xi / (f * k0 - kmup);
      r.i = rimu * ril1 / ril;
      r.ip = rimu * rip1 / ril;
    }
  }
  if (NEED_K) {
    double d0 = k0, d1 = k1;  // the recurrence in FP64 for both flavours, as for I above
    recur_up<double>((double)mu, (double)x, nl, -1.0, d0, d1);
    r.k = (T)d0;
    r.kp = (T)((double)(nu * xi) * d0 - d1);
  }
  return r;
}

}  // namespace tsb
