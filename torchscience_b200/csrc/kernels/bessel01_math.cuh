// J0 and J1 of real argument in FP64: the order-0/1 path behind bessel_j_0
// and behind bessel_j at ν = 0, ±1.
//
// The reference evaluates J0 with a rational approximation for x <= 5 and a
// modulus/phase rational form above (kernel/special_functions/bessel_j_0.h:91-129,
// bessel_j_1.h:91-130); bessel_j sends integer orders 0 and 1 there
// (bessel_j.h:240-316).  This path keeps that split between a small-argument
// fit and the modulus/phase form, with fits of its own (fits/gen_bessel01.py):
//
//   |x| < 1e-4: two Maclaurin terms.
//   |x| < X0 = 16.25π: one polynomial per interval of length π, each holding
//     exactly one zero z, in the form (x - z_hi - z_lo)·P(u).  The value
//     keeps full relative accuracy next to every zero below X0.
//   |x| >= X0: J_n = sqrt(2/(πx))·(P_n cos χ - Q_n sin χ), χ = x - (2n+1)π/4
//     (DLMF 10.17.3), P_n and x·Q_n polynomials in (X0/x)².  cos χ and sin χ
//     are formed from sin x and cos x, so no rounded multiple of π is
//     subtracted from x.
//
// Coefficient tables are read through the read-only data path, with the
// interval index fastest so a warp's lanes share cache lines.
#pragma once

#include <cuda_runtime.h>

#include "bessel01_fits.cuh"

namespace tsb {

struct J01 {
  double j0, j1;
};

namespace b01 {

constexpr double kInvPi = 0.31830988618379067;      // 1/π
constexpr double kInvSqrtPi = 0.56418958354775628;  // 1/sqrt(π)
constexpr int kB01Comp = 4;                         // compensated Horner steps

// UNROLL bounds how many coefficient loads are in flight (and held in
// registers) at once.
template <int ORDER, int UNROLL>
__device__ __forceinline__ double zero_form(double x, int i) {
  const double(*iv)[4] = ORDER == 0 ? fits::B01_J0_IV : fits::B01_J1_IV;
  const double(*cf)[fits::B01_NI] = ORDER == 0 ? fits::B01_J0_C : fits::B01_J1_C;
  const double u = (x - __ldg(&iv[i][0])) * __ldg(&iv[i][1]);
  double p = __ldg(&cf[fits::B01_DEG][i]);
#pragma unroll UNROLL
  for (int k = fits::B01_DEG - 1; k >= kB01Comp; --k) p = fma(p, u, __ldg(&cf[k][i]));
  // The last kB01Comp steps carry their rounding errors (the compensated
  // Horner scheme of Graillat, Langlois and Louvet, 2005: the product error
  // from an FMA, the sum error from TwoSum): their partial sums are as large
  // as the value, so they hold most of Horner's rounding near the interval
  // edges (|u| -> 1), where plain Horner measured up to 4 ulp.
  double c = 0.0;
#pragma unroll
  for (int k = kB01Comp - 1; k >= 0; --k) {
    const double a = __ldg(&cf[k][i]);
    const double pu = p * u, e1 = fma(p, u, -pu);
    const double s = pu + a, bb = s - pu, e2 = (pu - (s - bb)) + (a - bb);
    c = fma(c, u, e1 + e2);
    p = s;
  }
  // (x - z_hi) is exact near the zero (Sterbenz); (x - z_hi) - z_lo and the
  // product round once each
  return ((x - __ldg(&iv[i][2])) - __ldg(&iv[i][3])) * (p + c);
}

template <int N>
__device__ __forceinline__ double poly(const double (&c)[N], double w) {
  double p = c[N - 1];
#pragma unroll
  for (int k = N - 2; k >= 0; --k) p = fma(p, w, c[k]);
  return p;
}

}  // namespace b01

// J0(x), J1(x) for finite x (NEED0 / NEED1 select which are formed; the
// other field is left 0).  J0 is even and J1 odd in x.
template <bool NEED0, bool NEED1, int UNROLL = fits::B01_DEG>
__device__ __forceinline__ J01 bessel_j01(double x) {
  J01 r{0.0, 0.0};
  const double ax = fabs(x);
  if (ax < 1e-4) {  // two Maclaurin terms are exact to rounding (the next is below 2e-18 relative)
    r.j0 = fma(-0.25 * ax, ax, 1.0);
    r.j1 = 0.5 * ax * fma(-0.125 * ax, ax, 1.0);
  } else if (ax < fits::B01_X0) {
    const double q = ax * b01::kInvPi;
    if (NEED0) r.j0 = b01::zero_form<0, UNROLL>(ax, min(max((int)(q + 0.75), 1), fits::B01_NI - 1));
    if (NEED1) r.j1 = b01::zero_form<1, UNROLL>(ax, min((int)(q + 0.25), fits::B01_NI - 1));
  } else {
    const double rs = rsqrt(ax);  // 1/sqrt(x)
    const double r2 = rs * rs;    // 1/x
    const double w = fma(2.0 * fits::B01_X0_SQ * r2, r2, -1.0);  // 2(X0/x)² - 1
    double s, c;
    sincos(ax, &s, &c);
    const double amp = b01::kInvSqrtPi * rs;  // sqrt(2/(πx)) / sqrt(2)
    if (NEED0)  // cos χ0 = (c + s)/√2, sin χ0 = (s - c)/√2
      r.j0 = amp * (b01::poly(fits::B01_P0, w) * (c + s) - b01::poly(fits::B01_Q0, w) * r2 * (s - c));
    if (NEED1)  // cos χ1 = (s - c)/√2, sin χ1 = -(s + c)/√2
      r.j1 = amp * (b01::poly(fits::B01_P1, w) * (s - c) + b01::poly(fits::B01_Q1, w) * r2 * (s + c));
  }
  if (NEED1 && x < 0.0) r.j1 = -r.j1;
  return r;
}

#ifndef TSB_B01_UNROLL
#define TSB_B01_UNROLL 4
#endif
// Out of line and with bounded unrolling, for kernels that also hold the
// real-order evaluators: fully unrolled there, this path's table loads are
// scheduled early and raise the whole kernel's register count (105 -> 150
// for the FP64 J forward).
static __device__ __noinline__ J01 bessel_j01_call(double x) { return bessel_j01<true, true, TSB_B01_UNROLL>(x); }

}  // namespace tsb
