// Gamma-family evaluators: lnΓ, Γ, ψ, ψ', ψ'', ψ''' for the FP64 kernels
// (double) and the mixed kernels (float bulk, double where it is needed).
//
// Algorithms (published mathematics, not the reference's code):
//   - lnΓ and Γ: CUDA's lgamma/tgamma (called, not re-implemented), with
//     the reference's conventions at the poles (log_gamma.h:40-46: +inf at
//     the non-positive integers; gamma.h:84-87: +inf there as well).
//   - ψ^(n), n = 1..3: recurrence ψ^(n)(x) = ψ^(n)(x+1) - (-1)^n n!/x^(n+1)
//     up to a threshold, then the Bernoulli asymptotic series (DLMF 5.15.8,
//     5.11.2); for x <= 0 the reflection formulas (DLMF 5.15.6).  The shifted
//     sums are accumulated as one fraction num/den so the recurrence costs a
//     single division.
//   - ψ: the same asymptotic series for x >= 10 (8 in FP32); on [1, 2) the
//     factored fit (x - x0)·P(2x - 3) around the positive root x0 (fits.cuh,
//     generated by fits/gen_fits.py); other x reach [1, 2) by the recurrence;
//     reflection (DLMF 5.5.4) for x <= 0.
// The reference's own digamma/trigamma (digamma.h:10-25, trigamma.h:10-25)
// use a 3-term asymptotic after shifting to 6; their truncation error is
// about 1e-8, which the longer series here removes.
#pragma once

#include <math_constants.h>

#include "fits.cuh"

namespace tsb {

// Bernoulli numbers B_2 .. B_20.
#define TSB_B2 (1.0 / 6.0)
#define TSB_B4 (-1.0 / 30.0)
#define TSB_B6 (1.0 / 42.0)
#define TSB_B8 (-1.0 / 30.0)
#define TSB_B10 (5.0 / 66.0)
#define TSB_B12 (-691.0 / 2730.0)
#define TSB_B14 (7.0 / 6.0)
#define TSB_B16 (-3617.0 / 510.0)
#define TSB_B18 (43867.0 / 798.0)

__device__ __forceinline__ bool is_nonpos_int(double x) { return x <= 0.0 && x == floor(x); }
__device__ __forceinline__ bool is_nonpos_int(float x) { return x <= 0.0f && x == floorf(x); }

// ------------------------------------------------------------------ FP64
__device__ __forceinline__ double lgamma_d(double x) { return lgamma(x); }

__device__ __forceinline__ double gamma_d(double x) {
  if (is_nonpos_int(x)) return CUDART_INF;
  return tgamma(x);
}

template <typename T, int N>
__device__ __forceinline__ T horner(const T (&c)[N], T u) {
  T r = c[N - 1];
#pragma unroll
  for (int k = N - 2; k >= 0; --k) r = fma(r, u, c[k]);
  return r;
}

// ψ(x).  At the non-positive integers: -inf (the reference's upward
// recurrence divides by zero there, digamma.h:16-19).  On [1, 2) ψ is
// evaluated as (x - x0)·P(2x - 3) with x0 the positive root and P a fitted
// polynomial (fits.cuh), so it keeps full relative accuracy through the root;
// other x < 10 reach [1, 2) by the recurrence (one step up from (0, 1), or
// down from [2, 10) as a single fraction), x >= 10 uses the asymptotic series.
__device__ inline double digamma_d(double x) {
  if (isnan(x)) return x;
  if (isinf(x)) return x > 0.0 ? x : CUDART_NAN;
  double refl = 0.0;
  if (x <= 0.0) {
    if (x == floor(x)) return -CUDART_INF;
    double s, c;
    sincospi(x, &s, &c);
    refl = -CUDART_PI * c / s;  // ψ(x) = ψ(1-x) - π cot(πx)
    x = 1.0 - x;
  }
  if (x >= 10.0) {
    const double z = 1.0 / (x * x);
    const double tail =
        z * (TSB_B2 / 2 + z * (TSB_B4 / 4 + z * (TSB_B6 / 6 + z * (TSB_B8 / 8 + z * (TSB_B10 / 10 + z * (TSB_B12 / 12 + z * (TSB_B14 / 14 + z * (TSB_B16 / 16))))))));
    return refl + ((log(x) - 0.5 / x) - tail);
  }
  double acc = 0.0;
  if (x < 1.0) {
    acc = -1.0 / x;  // ψ(x) = ψ(x+1) - 1/x
    x += 1.0;
  } else if (x >= 2.0) {
    double num = 0.0, den = 1.0;  // ψ(x) = ψ(x-n) + Σ_{k=1..n} 1/(x-k)
    while (x >= 2.0) {
      x -= 1.0;
      num = fma(num, x, den);
      den *= x;
    }
    acc = num / den;
  }
  const double r = ((x - fits::PSI_X0_HI) - fits::PSI_X0_LO) * horner(fits::PSI_ROOT_D, fma(2.0, x, -3.0));
  return refl + (r + acc);
}

// ψ'(x).  +inf at the non-positive integers (trigamma.h:16-19 divides by 0).
__device__ inline double trigamma_d(double x) {
  if (isnan(x)) return x;
  if (isinf(x)) return x > 0.0 ? 0.0 : CUDART_NAN;
  double refl = 0.0, sign = 1.0;
  if (x <= 0.0) {
    if (x == floor(x)) return CUDART_INF;
    const double s = sinpi(x);
    refl = (CUDART_PI * CUDART_PI) / (s * s);  // ψ'(x) = π²/sin²(πx) - ψ'(1-x)
    sign = -1.0;
    x = 1.0 - x;
  }
  double num = 0.0, den = 1.0;  // Σ 1/(x+k)² as num/den
  while (x < 10.0) {
    const double x2 = x * x;
    num = fma(num, x2, den);
    den *= x2;
    x += 1.0;
  }
  const double r = 1.0 / x, z = r * r;
  const double asym =
      r + 0.5 * z + r * z * (TSB_B2 + z * (TSB_B4 + z * (TSB_B6 + z * (TSB_B8 + z * (TSB_B10 + z * (TSB_B12 + z * (TSB_B14 + z * (TSB_B16 + z * TSB_B18))))))));
  return refl + sign * (asym + num / den);
}

// ψ''(x) (tetragamma).
__device__ inline double tetragamma_d(double x) {
  if (isnan(x)) return x;
  if (isinf(x)) return x > 0.0 ? -0.0 : CUDART_NAN;
  double refl = 0.0, sign = 1.0;
  if (x <= 0.0) {
    if (x == floor(x)) return CUDART_NAN;
    // ψ''(1-x) - ψ''(x) = π d²/dx² cot(πx) = 2π³ cot csc²
    double s, c;
    sincospi(x, &s, &c);
    const double csc = 1.0 / s;
    refl = -2.0 * CUDART_PI * CUDART_PI * CUDART_PI * c * csc * csc * csc;  // ψ''(x) = ψ''(1-x) - 2π³cot·csc²
    sign = 1.0;
    x = 1.0 - x;
  }
  double num = 0.0, den = 1.0;  // Σ 1/(x+k)³
  while (x < 12.0) {
    const double x3 = x * x * x;
    num = fma(num, x3, den);
    den *= x3;
    x += 1.0;
  }
  // ψ''(x) ~ -[1/x² + 1/x³ + Σ_k B_2k (2k+1)/x^(2k+2)]
  const double r = 1.0 / x, z = r * r;
  const double asym =
      z + z * r + z * z * (TSB_B2 * 3 + z * (TSB_B4 * 5 + z * (TSB_B6 * 7 + z * (TSB_B8 * 9 + z * (TSB_B10 * 11 + z * (TSB_B12 * 13 + z * (TSB_B14 * 15 + z * (TSB_B16 * 17 + z * TSB_B18 * 19))))))));
  return refl + sign * (-asym - 2.0 * num / den);
}

// ψ'''(x) (pentagamma).
__device__ inline double pentagamma_d(double x) {
  if (isnan(x)) return x;
  if (isinf(x)) return x > 0.0 ? 0.0 : CUDART_NAN;
  double refl = 0.0, sign = 1.0;
  if (x <= 0.0) {
    if (x == floor(x)) return CUDART_INF;
    // ψ'''(x) + ψ'''(1-x) = -π d³/dx³ cot(πx) = 2π⁴ csc²(2cot² + csc²)
    double s, c;
    sincospi(x, &s, &c);
    const double csc2 = 1.0 / (s * s), cot = c / s;
    const double p4 = CUDART_PI * CUDART_PI * CUDART_PI * CUDART_PI;
    refl = 2.0 * p4 * csc2 * (2.0 * cot * cot + csc2);
    sign = -1.0;
    x = 1.0 - x;
  }
  double num = 0.0, den = 1.0;  // Σ 1/(x+k)⁴
  while (x < 12.0) {
    const double x2 = x * x, x4 = x2 * x2;
    num = fma(num, x4, den);
    den *= x4;
    x += 1.0;
  }
  // ψ'''(x) ~ 2/x³ + 3/x⁴ + Σ_k B_2k (2k+1)(2k+2)/x^(2k+3)
  const double r = 1.0 / x, z = r * r;
  const double asym =
      2.0 * z * r + 3.0 * z * z + z * z * r * (TSB_B2 * 12 + z * (TSB_B4 * 30 + z * (TSB_B6 * 56 + z * (TSB_B8 * 90 + z * (TSB_B10 * 132 + z * (TSB_B12 * 182 + z * (TSB_B14 * 240 + z * (TSB_B16 * 306 + z * TSB_B18 * 380))))))));
  return refl + sign * (asym + 6.0 * num / den);
}

// ------------------------------------------------------------------ mixed
// FP32 evaluators.  Arguments whose FP32 evaluation would lose accuracy
// (x <= 0: reflection and the negative roots; lnΓ near its zeros at 1 and 2)
// are classified into an FP64 region by the kernels in ops_gamma.cu; the
// guards here only keep the functions total when called directly.
__device__ __forceinline__ float lgamma_m(float x) {
  if (x <= 0.0f) return (float)lgamma_d((double)x);
  return lgammaf(x);
}

__device__ __forceinline__ float gamma_m(float x) {
  if (x <= 0.0f) return (float)gamma_d((double)x);
  return tgammaf(x);
}

__device__ inline float digamma_m(float x) {
  if (!(x > 0.0f)) return (float)digamma_d((double)x);
  if (isinf(x)) return x;
  if (x >= 8.0f) {
    const float z = 1.0f / (x * x);
    const float tail = z * ((float)(TSB_B2 / 2) + z * ((float)(TSB_B4 / 4) + z * ((float)(TSB_B6 / 6) + z * (float)(TSB_B8 / 8))));
    return (logf(x) - 0.5f / x) - tail;
  }
  float acc = 0.0f;
  if (x < 1.0f) {
    acc = -1.0f / x;
    x += 1.0f;
  } else if (x >= 2.0f) {
    float num = 0.0f, den = 1.0f;
    while (x >= 2.0f) {
      x -= 1.0f;
      num = fmaf(num, x, den);
      den *= x;
    }
    acc = num / den;
  }
  const float r = ((x - fits::PSI_X0_HI_F) - fits::PSI_X0_LO_F) * horner(fits::PSI_ROOT_F, fmaf(2.0f, x, -3.0f));
  return r + acc;
}

__device__ inline float trigamma_m(float x) {
  if (!(x > 0.0f)) return (float)trigamma_d((double)x);
  if (isinf(x)) return 0.0f;
  if (x < 1e-6f) return (float)trigamma_d((double)x);
  float num = 0.0f, den = 1.0f;
  while (x < 8.0f) {
    const float x2 = x * x;
    num = fmaf(num, x2, den);
    den *= x2;
    x += 1.0f;
  }
  const float r = 1.0f / x, z = r * r;
  const float asym = r + 0.5f * z + r * z * ((float)TSB_B2 + z * ((float)TSB_B4 + z * ((float)TSB_B6 + z * ((float)TSB_B8 + z * (float)TSB_B10))));
  return asym + num / den;
}

__device__ inline float tetragamma_m(float x) {
  if (!(x > 1e-3f)) return (float)tetragamma_d((double)x);
  if (isinf(x)) return -0.0f;
  float num = 0.0f, den = 1.0f;
  while (x < 10.0f) {
    const float x3 = x * x * x;
    num = fmaf(num, x3, den);
    den *= x3;
    x += 1.0f;
  }
  const float r = 1.0f / x, z = r * r;
  const float asym = z + z * r + z * z * ((float)(TSB_B2 * 3) + z * ((float)(TSB_B4 * 5) + z * ((float)(TSB_B6 * 7) + z * ((float)(TSB_B8 * 9) + z * (float)(TSB_B10 * 11)))));
  return -asym - 2.0f * num / den;
}

__device__ inline float pentagamma_m(float x) {
  if (!(x > 1e-2f)) return (float)pentagamma_d((double)x);
  if (isinf(x)) return 0.0f;
  float num = 0.0f, den = 1.0f;
  while (x < 10.0f) {
    const float x2 = x * x, x4 = x2 * x2;
    num = fmaf(num, x4, den);
    den *= x4;
    x += 1.0f;
  }
  const float r = 1.0f / x, z = r * r;
  const float asym = 2.0f * z * r + 3.0f * z * z + z * z * r * ((float)(TSB_B2 * 12) + z * ((float)(TSB_B4 * 30) + z * ((float)(TSB_B6 * 56) + z * ((float)(TSB_B8 * 90) + z * (float)(TSB_B10 * 132)))));
  return asym + 6.0f * num / den;
}

// Overloads so functors can be written once for T = double / float.
__device__ __forceinline__ double lgamma_t(double x) { return lgamma_d(x); }
__device__ __forceinline__ float lgamma_t(float x) { return lgamma_m(x); }
__device__ __forceinline__ double gamma_t(double x) { return gamma_d(x); }
__device__ __forceinline__ float gamma_t(float x) { return gamma_m(x); }
__device__ __forceinline__ double digamma_t(double x) { return digamma_d(x); }
__device__ __forceinline__ float digamma_t(float x) { return digamma_m(x); }
__device__ __forceinline__ double trigamma_t(double x) { return trigamma_d(x); }
__device__ __forceinline__ float trigamma_t(float x) { return trigamma_m(x); }
__device__ __forceinline__ double tetragamma_t(double x) { return tetragamma_d(x); }
__device__ __forceinline__ float tetragamma_t(float x) { return tetragamma_m(x); }
__device__ __forceinline__ double pentagamma_t(double x) { return pentagamma_d(x); }
__device__ __forceinline__ float pentagamma_t(float x) { return pentagamma_m(x); }

}  // namespace tsb
