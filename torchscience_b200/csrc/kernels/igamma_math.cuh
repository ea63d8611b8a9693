// Regularized incomplete gamma P(a,x), Q(a,x) = 1 - P and their first and
// second derivatives in a and x.
//
// Structure follows the reference's split (regularized_gamma_p.h:57-71):
// x < a + 1 uses the power series (regularized_gamma_p.h:11-27), otherwise
// the Legendre continued fraction for Q (regularized_gamma_p.h:29-55).  The
// rebuild differs in three ways, all from published mathematics:
//   1. the prefactor D = x^a e^{-x} / Γ(a+1) is formed as
//      a·log1pmx((x-a)/a) - ½ln(2πa) - μ(a) for a >= 10 (μ = Stirling
//      correction, DLMF 5.11.1), which avoids the a·ln x - lnΓ(a+1)
//      cancellation that limits the reference to ~1e-10 relative at a ~ 1e3;
//   2. the continued fraction runs as a forward (Wallis) recurrence,
//      renormalised each step, carrying d/da and d²/da² of the numerators
//      and denominators, so ∂P/∂a and ∂²P/∂a² are analytic (the reference
//      uses central differences, regularized_gamma_p_backward.h:19-25);
//   3. the series carries the harmonic sums H_n = Σ 1/(a+k) and
//      H2_n = Σ 1/(a+k)² for the same purpose.
// Iterations are capped (kIgammaMaxIter); inputs that would need more are
// evaluated to the cap (the result is then a truncated sum, never a hang).
#pragma once

#include "unconverged.cuh"
#include <math_constants.h>

#include "fits.cuh"
#include "gamma_math.cuh"
#include "temme_fits.cuh"

namespace tsb {

constexpr int kIgammaMaxIter = 2000;

template <typename T>
struct IgammaEps;
// Stopping tolerances: 2 ulp, so that convergents that jitter in the last
// bit (FMA contraction) still terminate.
template <>
struct IgammaEps<double> {
  static constexpr double v = 4.440892098500626e-16;
};
template <>
struct IgammaEps<float> {
  static constexpr float v = 2.3841858e-07f;
};

// log(1+t) - t, accurate for all t > -1.
__device__ inline double log1pmx_d(double t) {
  if (fabs(t) < 0.5) {
    // u = t/(2+t); log(1+t) - t = -t·u + 2u³(1/3 + u²/5 + u⁴/7 + ...)
    const double u = t / (2.0 + t), u2 = u * u;
    double s = 1.0 / 35.0;
#pragma unroll
    for (int k = 33; k >= 3; k -= 2) s = fma(s, u2, 1.0 / k);
    return fma(-t, u, 2.0 * u * u2 * s);
  }
  return log1p(t) - t;
}

// Stirling correction μ(a) = lnΓ(a) - [(a-½)ln a - a + ½ln 2π], a >= 10.
__device__ inline double stirling_mu_d(double a) {
  const double r = 1.0 / a, z = r * r;
  return r * (1.0 / 12 - z * (1.0 / 360 - z * (1.0 / 1260 - z * (1.0 / 1680 - z * (1.0 / 1188 - z * (691.0 / 360360 - z * (1.0 / 156)))))));
}

// Quantities of a alone and of x alone.  On a broadcast grid they are
// computed once per row / column (one value of a or x) into a table; an
// element then reads them instead of recomputing lnΓ, ψ and the logarithms.
// IgPre reads a table when it has one and computes the quantity otherwise,
// with the same expression, so both give identical results.
enum IgammaAuxA : int {
  kIgA_LG = 0,  // a < 10: lnΓ(a+1); a >= 10: ½ln(2πa) + μ(a)
  kIgA_LA,      // ln a
  kIgA_RA,      // 1/a
  kIgA_PSI,     // ψ(a)  (first and second derivatives)
  kIgA_PSI1,    // ψ'(a) (second derivatives)
  kIgA_F1,      // two floats in one slot: lgammaf(a+1) | __logf(a)      (classification)
  kIgA_F2,      // two floats in one slot: __logf(a+1) | float(ψ(a)+1/a) (classification, mixed routing)
  kIgAuxA
};
enum IgammaAuxX : int {
  kIgX_LX = 0,  // ln x
  kIgX_RX,      // 1/x
  kIgX_F1,      // __logf(x) in the slot's high half
  kIgAuxX
};

// The float table entries are packed two to a double slot and read as the
// slot's 32-bit halves, which costs no conversion instruction (a float
// stored as a double would be converted back on every element).
__device__ __forceinline__ double f2_pack(float hi, float lo) {
  return __hiloint2double(__float_as_int(hi), __float_as_int(lo));
}
__device__ __forceinline__ float f2_hi(double d) { return __int_as_float(__double2hiint(d)); }
__device__ __forceinline__ float f2_lo(double d) { return __int_as_float(__double2loint(d)); }

// A double split into floats hi + lo (|lo| <= ulp(hi)/2), for the mixed
// kernels' exponentials: ln D = a ln x - x - lnΓ(a+1) cancels by up to ~1e4
// in the benchmark domain, so it is formed in FP64 (igamma_lnd_mixed) and its
// exponential taken as exp(hi)(1 + lo) in float.
struct IgFF {
  float hi, lo;
};
__device__ __forceinline__ IgFF ff_split(double v) {
  const float hi = (float)v;
  return IgFF{hi, (float)(v - (double)hi)};
}
// exp(hi + lo) = exp(hi) (1 + lo) for |lo| << 1.
__device__ __forceinline__ float ff_exp(IgFF x) { return expf(x.hi) * (1.0f + x.lo); }

__device__ inline double igamma_lg(double a) {
  return a < 10.0 ? lgamma(a + 1.0) : 0.5 * log(2.0 * CUDART_PI * a) + stirling_mu_d(a);
}

template <int ORDER>
__device__ inline void igamma_aux_a(double a, double* o) {
  const float af = (float)a;
  o[kIgA_LG] = igamma_lg(a);
  o[kIgA_LA] = log(a);
  o[kIgA_RA] = 1.0 / a;
  o[kIgA_PSI] = ORDER >= 1 ? digamma_d(a) : 0.0;
  o[kIgA_PSI1] = ORDER >= 2 ? trigamma_d(a) : 0.0;
  o[kIgA_F1] = f2_pack(lgammaf(af + 1.0f), __logf(af));
  o[kIgA_F2] = f2_pack(__logf(af + 1.0f), (float)(o[kIgA_PSI] + o[kIgA_RA]));
}
__device__ inline void igamma_aux_x(double x, double* o) {
  o[kIgX_LX] = log(x);
  o[kIgX_RX] = 1.0 / x;
  o[kIgX_F1] = f2_pack(__logf((float)x), 0.0f);
}

struct IgPre {
  const double* A;  // table row for this a, or nullptr
  const double* X;  // table entry for this x, or nullptr
  double a, x;
  __device__ double lg() const { return A ? A[kIgA_LG] : igamma_lg(a); }
  __device__ double la() const { return A ? A[kIgA_LA] : log(a); }
  __device__ double ra() const { return A ? A[kIgA_RA] : 1.0 / a; }
  __device__ double psi() const { return A ? A[kIgA_PSI] : digamma_d(a); }
  __device__ double psi1() const { return A ? A[kIgA_PSI1] : trigamma_d(a); }
  __device__ float lgf() const { return A ? f2_hi(A[kIgA_F1]) : lgammaf((float)a + 1.0f); }
  __device__ float laf() const { return A ? f2_lo(A[kIgA_F1]) : __logf((float)a); }
  __device__ float la1f() const { return A ? f2_hi(A[kIgA_F2]) : __logf((float)a + 1.0f); }
  __device__ double lx() const { return X ? X[kIgX_LX] : log(x); }
  __device__ float prf() const { return A ? f2_lo(A[kIgA_F2]) : (float)(digamma_d(a) + 1.0 / a); }
  __device__ double rx() const { return X ? X[kIgX_RX] : 1.0 / x; }
  __device__ float lxf() const { return X ? f2_hi(X[kIgX_F1]) : __logf((float)x); }
};

// ln D(a,x), D = x^a e^{-x} / Γ(a+1).
// For a >= 10 the Temme form a·log1pmx(t) is used near x ~ a (|t| < 1/2);
// farther out log(x/a) is formed directly so that 1 + t = x/a does not lose
// the digits that t = (x-a)/a rounds away when x << a.
__device__ inline double igamma_log_prefix_d(double a, double x, const IgPre& P) {
  if (a < 10.0) return a * P.lx() - x - P.lg();
  const double t = (x - a) * P.ra();  // (x - a)/a to an ulp of t, which moves ln D by ~a t² 2^-53
  const double core = fabs(t) < 0.5 ? a * log1pmx_d(t) : a * log(x * P.ra()) - (x - a);
  return core - P.lg();
}

// ∂P/∂x = D·a/x from D = exp(lnD), or from its logarithm where D itself
// underflows (lnD < -700) but a/x lifts it back into range.
__device__ __forceinline__ double igamma_px_from(double D, double lnD, double a, const IgPre& P) {
  return lnD > -700.0 ? D * a * P.rx() : exp(lnD + (P.la() - P.lx()));
}

// Series S = Σ_{n>=0} x^n / ((a+1)...(a+n)) and its a-derivatives.
// ORDER 0: S; 1: + S1 = dS/da; 2: + S2 = d²S/da².
// Terms are produced four at a time from one reciprocal of
// (a+n+1)(a+n+2)(a+n+3)(a+n+4), which also yields the four 1/(a+n+k) that
// the harmonic sums H_n = Σ 1/(a+k), H2_n = Σ 1/(a+k)² need
// (dt_n/da = -t_n H_n, d²t_n/da² = t_n (H_n² + H2_n)).  Only used for
// x < a + 1, where the terms decrease monotonically.
template <typename TL, int ORDER>
__device__ inline void igamma_series(TL a, TL x, TL& S, TL& S1, TL& S2) {
  const TL eps = IgammaEps<TL>::v;
  const TL x2 = x * x;
  TL term = 1, sum = 1, H = 0, H2 = 0, s1 = 0, s2 = 0;
  TL e = a;
  for (int it = 0; it < kIgammaMaxIter / 4; ++it) {
    const TL e1 = e + TL(1), e2 = e + TL(2), e3 = e + TL(3), e4 = e + TL(4);
    e = e4;
    const TL p12 = e1 * e2, p34 = e3 * e4;
    const TL r = TL(1) / (p12 * p34);
    const TL tr = term * r;
    const TL t1 = tr * x * (e2 * p34);
    const TL t2 = tr * x2 * p34;
    const TL t3 = tr * (x2 * x) * e4;
    const TL t4 = tr * (x2 * x2);
    sum += (t1 + t2) + (t3 + t4);
    term = t4;
    bool done = t4 <= eps * sum;
    if (ORDER >= 1) {
      const TL r1 = r * (e2 * p34), r2 = r * (e1 * p34), r3 = r * (p12 * e4), r4 = r * (p12 * e3);
      const TL h1 = H + r1, h2 = h1 + r2, h3 = h2 + r3, h4 = h3 + r4;
      s1 -= (t1 * h1 + t2 * h2) + (t3 * h3 + t4 * h4);
      if (ORDER >= 2) {
        const TL q1 = H2 + r1 * r1, q2 = q1 + r2 * r2, q3 = q2 + r3 * r3, q4 = q3 + r4 * r4;
        s2 += (t1 * (h1 * h1 + q1) + t2 * (h2 * h2 + q2)) + (t3 * (h3 * h3 + q3) + t4 * (h4 * h4 + q4));
        H2 = q4;
        done = done && t4 * (h4 * h4 + q4) <= eps * s2;
      }
      H = h4;
      done = done && t4 * h4 <= eps * fabs(s1);
    }
    if (done) break;
  }
  // The last term still above the tolerance: the loop stopped at its cap.
  // (Checked on state that is live anyway; a loop-carried counter measured
  // ~10% slower on the benchmark grid.)
  if (!(term <= eps * sum)) note_unconverged();
  S = sum;
  S1 = s1;
  S2 = s2;
}

// Continued fraction G = b0 + a1/(b1 + a2/(b2 + ...)), b_n = x + 2n + 1 - a,
// a_n = -n(n - a), so that Q = x^a e^{-x}/Γ(a) / G.  Returns F = 1/G and its
// a-derivatives F1, F2 (ORDER as above).  The Wallis recurrences
//   A_n = b_n A_{n-1} + a_n A_{n-2}  (same for B)
// and their a-derivatives (b_n' = -1, a_n' = n) advance four steps between
// renormalisations by 1/B_n, which also give the convergent G_n = A_n / B_n.
template <typename TL, int ORDER>
__device__ inline void igamma_cf(TL a, TL x, TL& F, TL& F1, TL& F2) {
  const TL eps = IgammaEps<TL>::v;
  const TL b0 = x + TL(1) - a;
  TL Ap = 1, A = b0, Bp = 0, B = 1;
  TL dAp = 0, dA = -1, dBp = 0, dB = 0;
  TL ddAp = 0, ddA = 0, ddBp = 0, ddB = 0;
  TL G = b0, dG = -1, ddG = 0;
  int n = 0;
  for (int it = 0; it < kIgammaMaxIter / 4; ++it) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      ++n;
      const TL fn = TL(n);
      const TL an = -fn * (fn - a);
      const TL bn = b0 + TL(2) * fn;
      const TL An = bn * A + an * Ap;
      const TL Bn = bn * B + an * Bp;
      if (ORDER >= 2) {
        const TL ddAn = bn * ddA - TL(2) * dA + an * ddAp + TL(2) * fn * dAp;
        const TL ddBn = bn * ddB - TL(2) * dB + an * ddBp + TL(2) * fn * dBp;
        ddAp = ddA;
        ddA = ddAn;
        ddBp = ddB;
        ddB = ddBn;
      }
      if (ORDER >= 1) {
        const TL dAn = bn * dA - A + an * dAp + fn * Ap;
        const TL dBn = bn * dB - B + an * dBp + fn * Bp;
        dAp = dA;
        dA = dAn;
        dBp = dB;
        dB = dBn;
      }
      Ap = A;
      A = An;
      Bp = B;
      B = Bn;
    }
    const TL s = TL(1) / B;
    Ap *= s;
    Bp *= s;
    A *= s;
    B = TL(1);
    if (ORDER >= 1) {
      dAp *= s;
      dBp *= s;
      dA *= s;
      dB *= s;
    }
    if (ORDER >= 2) {
      ddAp *= s;
      ddBp *= s;
      ddA *= s;
      ddB *= s;
    }
    // Convergence of each quantity is judged against the size of the terms it
    // is formed from (dG = dA - A·dB can cancel, leaving rounding noise far
    // above 2 ulp of the result).
    const TL Gn = A;
    bool done = fabs(Gn - G) <= eps * fabs(Gn);
    G = Gn;
    if (ORDER >= 1) {
      const TL dGn = dA - A * dB;
      done = done && fabs(dGn - dG) <= eps * (fabs(dA) + fabs(A * dB));
      dG = dGn;
    }
    if (ORDER >= 2) {
      const TL ddGn = ddA - TL(2) * dA * dB - A * ddB + TL(2) * A * dB * dB;
      done = done && fabs(ddGn - ddG) <= eps * (fabs(ddA) + fabs(TL(2) * dA * dB) + fabs(A * ddB) + fabs(TL(2) * A * dB * dB));
      ddG = ddGn;
    }
    if (done) break;
  }
  if (n >= kIgammaMaxIter) note_unconverged();  // the step count reached the cap
  F = TL(1) / G;
  F1 = -dG * F * F;
  F2 = (TL(2) * dG * dG - G * ddG) * F * F * F;
}

// All quantities the forward / backward / double-backward kernels need.
struct IgammaOut {
  double p, q;       // P, Q
  double pa, px;     // ∂P/∂a, ∂P/∂x
  double paa, pax, pxx;
};

// Region ids shared by the classifier and the evaluators.  Besides the
// method (series / continued fraction / small-a / saturated), the series and
// continued-fraction regions are split by the ratio that sets their
// iteration count, so the lanes of a warp run loops of similar length.
enum IgammaRegion : int {
  // Numbered by decreasing cost (measured per element on B200), so that a
  // tile's sorted list starts with its most expensive groups.  The regions
  // are split by what sets their iteration count, so that the lanes of a warp
  // run loops of similar length: the ratio x/(a+1) and, next to the
  // transition x ~ a, where the term count grows like √a, the size of a
  // (kIgS3 / kIgC2 for a < 16, then the B, C, D buckets at 16, 64 and 256).
  // The mixed forward also buckets the a < 1 continued fractions, which it
  // runs in FP32 (kIgCa).
  kIgS3D = 0,        // series, x/(a+1) >= 0.7, a >= 256
  kIgC2D = 1,        // continued fraction, x/(a+1) <= 1.5, a >= 256
  kIgS3C = 2,        // as kIgS3D, 64 <= a < 256
  kIgC2C = 3,        // as kIgC2D, 64 <= a < 256
  kIgS3B = 4,        // as kIgS3D, 16 <= a < 64
  kIgC2B = 5,        // as kIgC2D, 16 <= a < 64
  kIgS3 = 6,         // series, 0.7 <= x/(a+1) < 1, a < 16
  kIgC2 = 7,         // continued fraction, x/(a+1) <= 1.5, a < 16
  kIgC1 = 8,         // continued fraction, x/(a+1) > 1.5
  kIgS2 = 9,         // series, x/(a+1) < 0.7
  kIgC0 = 10,        // continued fraction, 3 < x/(a+1) <= 10
  kIgCa = 11,        // mixed forward only: continued fraction, a < 1 (FP32 there)
  kIgS1 = 12,        // series, x/(a+1) < 0.35
  kIgS0 = 13,        // series, 0.01 <= x/(a+1) < 0.1
  kIgSmallA = 14,    // a < 1, 0.1 (a+1) <= x < a + 1: series for P, dedicated formula for Q
  kIgC00 = 15,       // continued fraction, x/(a+1) > 10
  kIgS00 = 16,       // series, x/(a+1) < 0.01
  kIgSmallA0 = 17,   // a < 1, x < 0.1 (a+1)
  kIgSat1 = 18,      // Q and every derivative underflow to 0 (P = 1)
  kIgSat0 = 19,      // P and every derivative underflow to 0 (Q = 1)
  kIgSpecial = 20,   // NaN / domain / x == 0 / x == inf
  kIgRegions = 21
};

// The transition regions (kIgS3 for the series, kIgC2 for the continued
// fraction) bucketed by the size of a.
__device__ __forceinline__ int igamma_transition_bucket(bool cf, float a) {
  const int base = a >= 256.0f ? kIgS3D : a >= 64.0f ? kIgS3C : a >= 16.0f ? kIgS3B : kIgS3;
  return base + (cf ? 1 : 0);
}

// Regions whose loops are short enough for FP32 accumulation (mixed kernels).
__device__ __forceinline__ bool igamma_fp32_ok(int region) {
  return region == kIgS00 || region == kIgS0 || region == kIgS1 || region == kIgC00 || region == kIgC0 ||
         region == kIgCa;
}

// Region of (a, x) from cheap float arithmetic.
// MIXED_FWD: the mixed forward's bucket kIgCa; the other kernels bucket
// those elements by iteration count.
__device__ __forceinline__ int igamma_classify(double ad, double xd, const IgPre& P, bool mixed_fwd = false) {
  if (!(xd >= 0.0) || !(ad > 0.0) || xd == 0.0 || isinf(xd) || isinf(ad)) return kIgSpecial;
  const float a = (float)ad, x = (float)xd;
  if (!(a > 0.0f) || !(x > 0.0f) || isinf(a) || isinf(x)) return kIgSpecial;
  // float estimate of ln D
  const float lnd = a * P.lxf() - x - P.lgf();
  // Saturation: the prefactor (and ∂P/∂x = D·a/x, whose ratio a/x is
  // included) is below e^-760, so in double P or Q and all derivatives are 0.
  // The float estimate's absolute error grows like a·ln x·2^-24; up to
  // a = 1e5 it stays far inside the 15-unit margin to the double underflow
  // threshold e^-745.  Larger a (or x) skip the test: the FP64 evaluator
  // forms ln D accurately and saturates there.
  const bool can_saturate = a < 1e5f && x < 1e5f;
  // ln(a/x) and the ratio λ = x/(a+1) without divisions: the logarithms come
  // from the tables, and λ is compared as x against multiples of a + 1
  const float lratio = fmaxf(0.0f, P.laf() - P.lxf());
  const float a1 = a + 1.0f;
  if (x < a1) {
    // P <= D·(a+1)/(a+1-x) ~ D·a.
    if (can_saturate && lnd + P.la1f() + lratio < -760.0f) return kIgSat0;
    if (a < 1.0f) return x < 0.1f * a1 ? kIgSmallA0 : kIgSmallA;
    return x < 0.01f * a1 ? kIgS00 : x < 0.1f * a1 ? kIgS0 : x < 0.35f * a1 ? kIgS1 : x < 0.7f * a1 ? kIgS2
                                                                                : igamma_transition_bucket(false, a);
  }
  // Q = a D F with F <= 1/(x+1-a) <= 1.
  if (can_saturate && lnd + P.laf() + lratio < -760.0f) return kIgSat1;
  if (mixed_fwd && a < 1.0f) return kIgCa;
  return x > 10.0f * a1 ? kIgC00 : x > 3.0f * a1 ? kIgC0 : x > 1.5f * a1 ? kIgC1 : igamma_transition_bucket(true, a);
}
__device__ __forceinline__ int igamma_classify(double ad, double xd, bool mixed_fwd = false) {
  return igamma_classify(ad, xd, IgPre{nullptr, nullptr, ad, xd}, mixed_fwd);
}

// Q(a, x) for a < 1, x < a + 1 without the 1 - P cancellation (P -> 1 as
// a -> 0): from γ(a,x) = Σ (-1)^n x^(a+n) / (n!(a+n)),
//   Q = -expm1(a ln x - lnΓ(1+a)) - x^a/Γ(1+a) · a · Σ_{n>=1} (-x)^n / (n!(a+n)),
// with lnΓ(1+a) = a·G(2a-1) from the fit in fits.cuh (no rounding of 1 + a).
__device__ inline double igamma_q_small_a_d(double a, double x, double lx) {
  const double lg1p = a * horner(fits::LGAMMA1P_D, fma(2.0, a, -1.0));
  const double e = a * lx - lg1p;
  double term = 1.0, T = 0.0;
  {  // counted loop: reaching the cap is recorded (note_unconverged)
    int n = 1;
    for (; n < 80; ++n) {
      term *= -x / (double)n;
      const double t = term / (a + (double)n);
      T += t;
      if (fabs(t) <= 1e-17 * fabs(T)) break;
    }
    if (n >= 80) note_unconverged();
  }
  return -expm1(e) - exp(e) * a * T;
}

// Temme's uniform asymptotic expansion (DLMF 8.12.3-8.12.4, 8.12.10), for
// a >= TEMME_A_MIN and TEMME_LAM_LO <= x/a <= TEMME_LAM_HI: the transition
// x ~ a, where the series and the continued fraction need a number of terms
// growing like √a, in a fixed number of operations.  With u = x/a - 1 and
// η = sign(u) sqrt(-2 (ln(1+u) - u)),
//   Q = ½ erfc(η sqrt(a/2)) + R,  P = ½ erfc(-η sqrt(a/2)) - R,
//   R = e^(-aη²/2) / sqrt(2πa) · S,  S = Σ c_k(η) a^-k,
// the smaller of P and Q computed directly and the other as 1 minus it.
// The c_k are Taylor series in η (temme_fits.cuh, generated and checked
// against mpmath by fits/gen_temme.py).  First derivatives: ∂P/∂x = D a/x with
// D = e^(-aη²/2) / (sqrt(2πa) Γ*(a)), Γ*(a) = e^μ(a) (DLMF 5.11.3); with
// dη/da = -(u/η)/a,
//   ∂P/∂a = e^(-aη²/2)/sqrt(2πa) · [η/2 - u/η - S (ln(1+u) - 1/(2a)) + (Sk + Se u/η)/a],
// Se = Σ c_k'(η) a^-k, Sk = Σ k c_k(η) a^-k.
__device__ __forceinline__ bool igamma_temme_applies(double a, double x) {
  return a >= fits::TEMME_A_MIN && x >= fits::TEMME_LAM_LO * a && x <= fits::TEMME_LAM_HI * a;
}

// Out of line: one copy per kernel, fetched only by the warps that take it
// (the kernels that call it are bound by instruction fetch, and its sums are
// a few hundred straight-line FMAs).
template <int ORDER>
__device__ __noinline__ IgammaOut igamma_temme_d(double a, double x, const IgPre P) {
  IgammaOut o;
  o.pa = o.px = o.paa = o.pax = o.pxx = 0.0;
  const double r = P.ra();
  const double u = (x - a) * r;
  const double lm = log1pmx_d(u);  // ln(1+u) - u = -η²/2
  const double eta = u == 0.0 ? 0.0 : copysign(sqrt(-2.0 * lm), u);
  double S, Se, Sk;
  fits::temme_sums<(ORDER >= 1)>(eta, r, S, Se, Sk);
  const double pref = exp(fma(a, lm, -0.5 * (1.8378770664093453 + P.la())));  // e^(-aη²/2) / sqrt(2πa)
  const double s = eta * sqrt(0.5 * a);
  const double R = pref * S;
  if (eta >= 0.0) {
    o.q = fma(0.5, erfc(s), R);
    o.p = 1.0 - o.q;
  } else {
    o.p = fma(0.5, erfc(-s), -R);
    o.q = 1.0 - o.p;
  }
  if (ORDER >= 1) {
    const double rue = eta == 0.0 ? 1.0 : u / eta;
    o.pa = pref * (0.5 * eta - rue - S * (log1p(u) - 0.5 * r) + r * fma(Se, rue, Sk));
    // D a/x = pref e^-μ / (1+u); e^-μ by its Taylor series (μ <= 1/(12 a) <= 0.0042)
    const double mu = stirling_mu_d(a);
    double em = 1.0;  // 1 - μ(1 - μ/2(1 - μ/3(...))), seven terms: the rest is below 1e-20
#pragma unroll
    for (int k = 7; k >= 1; --k) em = fma(-mu * (1.0 / k), em, 1.0);
    o.px = pref * em / (1.0 + u);
  }
  return o;
}

// FP64 evaluation.  ORDER 0: p,q; 1: + pa, px; 2: + paa, pax, pxx.
// WANT_Q: Q is requested (selects the small-a formula for Q where it matters).
// UNIFORM: the uniform expansion takes its window (ORDER <= 1).  The callers
// without per-row / per-column tables (the map kernel: independent points)
// set it; the row-sorted sweep does not, because there the expansion's call
// site alone measured slower for every element than the series it replaces
// for the ~2% in its window (the sweep is bound by instruction fetch).
template <int ORDER, bool WANT_Q = false, bool UNIFORM = false>
__device__ inline IgammaOut igamma_eval_d(double a, double x, const IgPre& P) {
  IgammaOut o;
  o.pa = o.px = o.paa = o.pax = o.pxx = 0.0;
  if (isnan(a) || isnan(x) || x < 0.0 || a <= 0.0) {
    o.p = o.q = CUDART_NAN;
    o.pa = o.px = o.paa = o.pax = o.pxx = CUDART_NAN;
    return o;
  }
  if (x == 0.0) {
    o.p = 0.0;
    o.q = 1.0;
    return o;
  }
  if (isinf(x)) {
    o.p = 1.0;
    o.q = 0.0;
    return o;
  }
  if (isinf(a)) {
    o.p = 0.0;
    o.q = 1.0;
    return o;
  }
  if (UNIFORM && ORDER <= 1 && igamma_temme_applies(a, x)) return igamma_temme_d<ORDER>(a, x, P);
  const double lnD = igamma_log_prefix_d(a, x, P);
  const double lx = P.lx();
  // ∂P/∂x = x^(a-1) e^{-x} / Γ(a) = D·a/x
  if (x < a + 1.0) {
    // P <= D (a+1): below e^-760 it underflows (ln(a+1) from the table's float
    // value: the test has a margin of 15 to the underflow threshold e^-745)
    if (lnD + (double)P.la1f() < -760.0) {
      o.p = 0.0;
      o.q = 1.0;
      return o;
    }
    double psi_a = 0.0, psi1_a = 0.0;
    if (ORDER >= 1) psi_a = P.psi();
    if (ORDER >= 2) psi1_a = P.psi1();
    double S, S1 = 0.0, S2 = 0.0;
    igamma_series<double, ORDER>(a, x, S, S1, S2);
    const double D = exp(lnD);
    o.p = D * S;
    o.q = (WANT_Q && a < 1.0) ? igamma_q_small_a_d(a, x, lx) : 1.0 - o.p;
    if (ORDER >= 1) {
      const double ra = P.ra();
      const double L1 = lx - (psi_a + ra);  // d lnD/da = ln x - ψ(a+1)
      o.pa = D * fma(L1, S, S1);
      o.px = igamma_px_from(D, lnD, a, P);
      if (ORDER >= 2) {
        const double L2 = -(psi1_a - ra * ra);  // -ψ'(a+1)
        o.paa = D * ((L2 + L1 * L1) * S + 2.0 * L1 * S1 + S2);
        o.pax = o.px * (lx - psi_a);
        o.pxx = o.px * ((a - 1.0) / x - 1.0);
      }
    }
  } else {
    const double lnE = lnD + P.la();  // E = x^a e^{-x}/Γ(a)
    if (lnE < -760.0) {
      o.p = 1.0;
      o.q = 0.0;
      return o;
    }
    double psi_a = 0.0, psi1_a = 0.0;
    if (ORDER >= 1) psi_a = P.psi();
    if (ORDER >= 2) psi1_a = P.psi1();
    double F, F1 = 0.0, F2 = 0.0;
    igamma_cf<double, ORDER>(a, x, F, F1, F2);
    const double E = exp(lnE);
    o.q = E * F;
    o.p = 1.0 - o.q;
    if (ORDER >= 1) {
      const double E1 = lx - psi_a;
      const double qa = E * fma(E1, F, F1);
      o.pa = -qa;
      o.px = lnE > -700.0 ? E * P.rx() : exp(lnE - lx);  // E/x
      if (ORDER >= 2) {
        const double E2 = -psi1_a;
        o.paa = -E * ((E2 + E1 * E1) * F + 2.0 * E1 * F1 + F2);
        o.pax = o.px * E1;
        o.pxx = o.px * ((a - 1.0) / x - 1.0);
      }
    }
  }
  return o;
}

// Mixed evaluation of P or Q alone (the forward) in the light regions
// (igamma_fp32_ok), entirely in FP32: ln D in float-float from the double
// per-row / per-column quantities (the tables, or computed here), D =
// exp(hi)(1 + lo), and the series or continued fraction in float.  In these
// regions x < 0.35 (a+1) or x > 3 (a+1) (or a < 1 for the continued
// fraction), so for a >= 10 the prefactor is always the direct form
// a (ln x - ln a) - (x - a) - C(a).  The float continued fraction carries
// ~1e-6 relative error in Q, which P = 1 - Q scales down by Q/P < 1 in these
// regions; Q itself takes the FP64 continued fraction.
// ln D for the mixed evaluators, in FP64 from the per-row / per-column double
// quantities (a few FP64 operations, far fewer issue slots than the same
// sum in float-float arithmetic): a ln x - x - lnΓ(a+1) for a < 10, else the
// direct form a (ln x - ln a) - (x - a) - C(a) (these regions keep x away
// from a).  Its absolute error, ~1e-16 times the terms' size, is far below
// what the float evaluation needs.
__device__ __forceinline__ double igamma_lnd_mixed(float a, float x, const IgPre& P) {
  const double ad = a, xd = x;
  return a < 10.0f ? fma(ad, P.lx(), -xd) - P.lg() : fma(ad, P.lx() - P.la(), -(xd - ad)) - P.lg();
}

template <bool WANT_Q>
__device__ inline IgammaOut igamma_eval_mf(int region, float a, float x, const IgPre& P) {
  IgammaOut o;
  o.pa = o.px = o.paa = o.pax = o.pxx = 0.0;
  const double lnDd = igamma_lnd_mixed(a, x, P);
  const IgFF lnD = ff_split(lnDd);
  if (region != kIgC0 && region != kIgC00 && region != kIgCa) {
    float S, S1, S2;
    igamma_series<float, 0>(a, x, S, S1, S2);
    const float pv = ff_exp(lnD) * S;
    o.p = pv;
    o.q = 1.0 - (double)pv;
  } else {
    double F;
    if (WANT_Q) {
      double F1, F2;
      igamma_cf<double, 0>((double)a, (double)x, F, F1, F2);
    } else {
      float f, f1, f2;
      igamma_cf<float, 0>(a, x, f, f1, f2);
      F = f;
    }
    o.q = (double)ff_exp(ff_split(lnDd + P.la())) * F;  // E F, E = D a
    o.p = 1.0 - o.q;
  }
  return o;
}

// exp(v)·m in float, for ln-values v (float-float) whose exponential is
// below the normal range: expf is taken at v + 64 and the product scaled by
// e^-64 last, so a subnormal result is rounded once.
__device__ __forceinline__ float ff_exp_mul(IgFF v, float m) {
  if (v.hi > -80.0f) return expf(v.hi) * (1.0f + v.lo) * m;
  return (expf(v.hi + 64.0f) * (1.0f + v.lo) * m) * 1.60381089e-28f;
}
// The same for several factors of one exponential: exp(v) = m·s, and
// ff_exp_apply(e, f) = (m·f)·s rounds exactly as ff_exp_mul(v, f) does.
struct IgFFExp {
  float m, s;
};
__device__ __forceinline__ IgFFExp ff_exp_split(IgFF v) {
  if (v.hi > -80.0f) return IgFFExp{expf(v.hi) * (1.0f + v.lo), 1.0f};
  return IgFFExp{expf(v.hi + 64.0f) * (1.0f + v.lo), 1.60381089e-28f};
}
__device__ __forceinline__ float ff_exp_apply(IgFFExp e, float f) { return (e.m * f) * e.s; }

// Regions whose first derivatives the mixed kernels evaluate in FP32 (bit r
// for region r); the others, and every second derivative, run in FP64.
// Measured against the FP64 kernels on the 4096 x 4096 benchmark grid (max
// relative error of P, ∂P/∂a, ∂P/∂x): the series regions up to x < 0.7 (a+1)
// stay below 5e-7; kIgS3 reaches 3e-6, the float continued fraction's
// a-derivative 1.4e-6 (kIgC0) to 5.5e-6 (kIgC2); kIgSmallA 1.5e-6 where
// ln x > ψ(a+1) (those elements take FP64).  The fraction regions run in
// FP32 only through the large-x expansion (igamma_asym_f, x >= 20).
#ifndef TSB_IG_FP32_MASK1
#define TSB_IG_FP32_MASK1 ((1u << kIgS00) | (1u << kIgS0) | (1u << kIgS1) | (1u << kIgS2) | (1u << kIgC00) | \
                           (1u << kIgC0) | (1u << kIgSmallA0) | (1u << kIgSmallA))
#endif

// Γ(a,x) x^(1-a) e^x = Σ_{k>=0} (a-1)(a-2)...(a-k) / x^k, the large-x
// expansion (DLMF 8.11.2), in float, with its a-derivative: t_k = t_{k-1}
// (a-k)/x and dt_k/da = (dt_{k-1}/da)(a-k)/x + t_{k-1}/x, products only.
// For x >= 20 and x >= 3(a+1) the terms fall below 3e-8 of the sum within
// about 15 terms (they shrink by (a-k)/x <= 1/3 while k < a, and by at most
// k/x beyond, the smallest being ~2e-8 at x = 20); an integer a ends the
// value's series exactly.  The derivative enters ∂Q/∂a as E1 S + S1 with S ~ 1
// and E1 = ln x - ψ(a) >= ~2.5 here, so its terms are judged against
// dscale = E1, not against S1 (~1/x), whose own relative accuracy does not
// matter.  The loop also stops at the smallest term once the terms grow (the
// expansion diverges beyond k ~ x + a).
__device__ inline void igamma_asym_f(float a, float x, float dscale, float& S, float& S1) {
  const float rx = 1.0f / x;
  float t = 1.0f, dt = 0.0f;
  S = 1.0f;
  S1 = 0.0f;
  for (int k = 1; k <= 48; ++k) {
    const float f = (a - (float)k) * rx;
    if ((float)k > a && fabsf(f) >= 1.0f) break;  // terms would grow
    dt = fmaf(dt, f, t * rx);
    t *= f;
    S += t;
    S1 += dt;
    if (fabsf(t) <= 3e-8f * S && fabsf(dt) <= 3e-8f * dscale) break;
  }
}

// Mixed evaluation of P (or Q) with ∂P/∂a and ∂P/∂x, entirely in FP32, for
// float data in the regions of TSB_IG_FP32_MASK1.
//   ln D = a ln x - x - lnΓ(a+1) (a < 10) or a (ln x - ln a) - (x - a) - C(a)
//   in float-float from the double per-row / per-column quantities, exact to
//   ~1e-11 absolute even where the terms cancel;
//   series (x < a+1):  P = D S,  ∂P/∂a = D (L1 S + S1),  L1 = ln x - ψ(a+1);
//   fraction:          Q = E F,  ∂Q/∂a = E (E1 F + F1),  E = D a,
//                      E1 = ln x - ψ(a) (L1 and E1 in float-float from the
//                      tables, so their cancellation near x ~ a costs nothing);
//   ∂P/∂x = D a / x = E / x from its logarithm, in range wherever the result is.
// In the series region L1 S and S1 have the same sign for x <= a and nearly
// so up to a + 1, and in the fraction region E1 > 0 and F1 > 0: the
// derivative sums do not cancel.  Q in the series region (and P in the
// fraction region) is 1 - the other, in double.  Small a with Q requested
// keeps the FP64 small-a formula (the caller routes it there).
template <bool WANT_Q>
__device__ inline IgammaOut igamma_eval_mf1(int region, float a, float x, const IgPre& P) {
  IgammaOut o;
  o.paa = o.pax = o.pxx = 0.0;
  const double lnDd = igamma_lnd_mixed(a, x, P), lnEd = lnDd + P.la();
  const IgFF lnD = ff_split(lnDd), lnE = ff_split(lnEd);
  const IgFF lnEx = ff_split(lnEd - P.lx());  // ln(E/x) = ln ∂P/∂x
  // one exponential per distinct exponent: ∂P/∂x shares ln(E/x) with the
  // expansion's value and a-derivative; the series and the fraction take a
  // second one, of ln D or ln E
  const IgFFExp ex = ff_exp_split(lnEx);
  o.px = ff_exp_apply(ex, 1.0f);
  if (region == kIgC0 || region == kIgC00) {
    // Q = (E/x) S, ∂Q/∂a = (E/x) (E1 S + S1), E1 = ln x - ψ(a) (x >= 20 here)
    float S, S1;
    const IgFF E1 = ff_split(P.lx() - P.psi());
    igamma_asym_f(a, x, fabsf(E1.hi), S, S1);
    const float qv = ff_exp_apply(ex, S);
    o.q = qv;
    o.p = 1.0 - (double)qv;
    o.pa = -(double)ff_exp_apply(ex, fmaf(E1.hi, S, fmaf(E1.lo, S, S1)));
  } else if (region != kIgC1 && region != kIgC2) {
    float S, S1, S2;
    igamma_series<float, 1>(a, x, S, S1, S2);
    const IgFF L1 = ff_split(P.lx() - (P.psi() + P.ra()));
    const IgFFExp ed = ff_exp_split(lnD);
    const float pv = ff_exp_apply(ed, S);
    o.p = pv;
    o.q = 1.0 - (double)pv;
    o.pa = ff_exp_apply(ed, fmaf(L1.hi, S, fmaf(L1.lo, S, S1)));
  } else {
    float F, F1, F2;
    igamma_cf<float, 1>(a, x, F, F1, F2);
    const IgFF E1 = ff_split(P.lx() - P.psi());
    const IgFFExp ee = ff_exp_split(lnE);
    const float qv = ff_exp_apply(ee, F);
    o.q = qv;
    o.p = 1.0 - (double)qv;
    o.pa = -(double)ff_exp_apply(ee, fmaf(E1.hi, F, fmaf(E1.lo, F, F1)));
  }
  return o;
}

// Whether the mixed kernels evaluate (a, x) of `region` with its first
// derivatives in FP64: regions outside TSB_IG_FP32_MASK1; the small-a Q;
// ln x > ψ(a+1) in kIgSmallA (there L1 S and S1 have opposite signs); the
// fraction regions below x = 20 (the expansion needs x >= 20).
__device__ __forceinline__ bool igamma_needs_fp64_1(int region, float xf, const IgPre& P, bool want_q) {
  return region == kIgSpecial || !((TSB_IG_FP32_MASK1 >> region) & 1u) ||
         (want_q && (region == kIgSmallA || region == kIgSmallA0)) ||
         (region == kIgSmallA && P.lxf() > P.prf()) || ((region == kIgC0 || region == kIgC00) && !(xf >= 20.0f));
}

// The FP64 evaluation with first derivatives as one out-of-line function,
// for the mixed kernels' FP64 regions.
template <bool WANT_Q, bool UNIFORM>
__device__ __noinline__ IgammaOut igamma_eval_d1_call(float a, float x, const IgPre P) {
  return igamma_eval_d<1, WANT_Q, UNIFORM>((double)a, (double)x, P);
}

// Evaluation for float data.  P or Q alone (ORDER 0): FP32 in the light
// regions (igamma_eval_mf), FP64 elsewhere: the heavy regions (large a near
// the transition x ~ a, where the term count grows like √a and float
// accumulation would exceed 1e-6) and the small-a Q.  First derivatives
// (ORDER 1): FP32 in the regions of TSB_IG_FP32_MASK1 (igamma_eval_mf1), FP64
// elsewhere.  Second derivatives: FP64.
template <int ORDER, bool WANT_Q = false, bool UNIFORM = false>
__device__ inline IgammaOut igamma_eval_m(int region, float af, float xf, const IgPre& P) {
  if constexpr (ORDER >= 2) {
    return igamma_eval_d<ORDER, WANT_Q>((double)af, (double)xf, P);
  } else if constexpr (ORDER == 1) {
    // The FP64 evaluator is one out-of-line copy (igamma_eval_d1_call), so
    // the inline code is the FP32 path.
    if (igamma_needs_fp64_1(region, xf, P, WANT_Q)) return igamma_eval_d1_call<WANT_Q, UNIFORM>(af, xf, P);
    return igamma_eval_mf1<WANT_Q>(region, af, xf, P);
  } else {
    if (region == kIgSmallA || region == kIgSmallA0) {
      if (WANT_Q) return igamma_eval_d<0, true, UNIFORM>((double)af, (double)xf, P);
      region = kIgS1;
    }
    if (!igamma_fp32_ok(region)) return igamma_eval_d<0, WANT_Q, UNIFORM>((double)af, (double)xf, P);
    return igamma_eval_mf<WANT_Q>(region, af, xf, P);
  }
}

__device__ __forceinline__ IgammaOut igamma_saturated(bool upper_is_zero) {
  IgammaOut o;
  o.p = upper_is_zero ? 1.0 : 0.0;
  o.q = 1.0 - o.p;
  o.pa = o.px = o.paa = o.pax = o.pxx = 0.0;
  return o;
}

template <int ORDER, bool WANT_Q = false, bool UNIFORM = false>
__device__ __forceinline__ IgammaOut igamma_eval(int region, double a, double x, const IgPre& P) {
  if (region == kIgSat0 || region == kIgSat1) return igamma_saturated(region == kIgSat1);
  return igamma_eval_d<ORDER, WANT_Q, UNIFORM>(a, x, P);
}
template <int ORDER, bool WANT_Q = false, bool UNIFORM = false>
__device__ __forceinline__ IgammaOut igamma_eval(int region, float a, float x, const IgPre& P) {
  if (region == kIgSat0 || region == kIgSat1) return igamma_saturated(region == kIgSat1);
  return igamma_eval_m<ORDER, WANT_Q, UNIFORM>(region, a, x, P);
}
// Without tables (map-kernel callers of independent points): the uniform
// expansion takes its window.
template <int ORDER, bool WANT_Q = false, typename T>
__device__ __forceinline__ IgammaOut igamma_eval(int region, T a, T x) {
  return igamma_eval<ORDER, WANT_Q, true>(region, a, x, IgPre{nullptr, nullptr, (double)a, (double)x});
}

}  // namespace tsb
