// Regularized incomplete beta I_x(a, b) in FP64 with its derivatives: the
// functors of incomplete_beta, incomplete_beta_backward and
// incomplete_beta_backward_backward.
//
// Reference behaviour (kernel/special_functions/incomplete_beta.h:27-63,
// incomplete_beta_backward.h:212-276, incomplete_beta_backward_backward.h:110-237):
//   forward:  NaN if a <= 0 or b <= 0; 0 for x <= 0; 1 for x >= 1; x when
//             a = b = 1; 1 - (1-x)^b when a = 1; x^a when b = 1; otherwise
//             I_x(a, b) = 1 - I_(1-x)(b, a) when x > (a+1)/(a+b+2), else
//             x^a (1-x)^b / (a B(a, b)) times the continued fraction
//             (DLMF 8.17.22), evaluated by modified Lentz with 200 terms.
//   backward: zeros for x <= 0 or x >= 1 (checked before a, b); NaN for
//             a <= 0 or b <= 0; ∂x = the beta density; ∂a, ∂b as
//             log-weighted integrals of the density, by adaptive
//             Gauss–Kronrod quadrature (tolerance 1e-12).
//   double backward: the same conventions; second derivatives from
//             log- and log²-weighted integrals.
//
// Here the continued fraction is run by the Wallis recurrences A_n, B_n
// together with their derivatives in the two parameters (each d_n is a
// rational function of p and q), rescaled by 1/B_n every step, so
//   J = I_y(p, q) = exp(p ln y + q ln(1-y) - ln B(p, q) - ln p) / K,
//   ∂J/∂p = J (ln y - [ψ(p) - ψ(p+q)] - 1/p - K_p/K),
//   ∂J/∂q = J (ln(1-y) - [ψ(q) - ψ(p+q)] - K_q/K),
// with ln B from Stirling's form and the ψ differences without cancellation
// (beta_math.cuh).  The a/b derivatives are exact to rounding instead of to
// a quadrature tolerance, and the fraction runs to convergence (up to 4000
// terms) rather than a fixed 200.  The second derivatives in x are
// analytic; ∂²/∂a², ∂²/∂a∂b and ∂²/∂b² are central differences of the
// analytic first derivatives with step ε^(1/3)·a (or ·b).
#pragma once

#include "unconverged.cuh"
#include <math_constants.h>

#include "beta_math.cuh"
#include "dispatch.cuh"

namespace tsb {

struct IbetaOut {
  double v, dx, da, db;
};

namespace ib {
constexpr int kMaxPairs = 2000;                    // 4000 terms of the fraction
constexpr double kTol = 4e-16;                     // convergence of K between pairs of terms
constexpr double kTolD = 1e-15;                    // convergence of K_p, K_q (scaled, below)
constexpr double kStep = 6.0554544523933395e-06;  // ε^(1/3): relative step of the differences
}  // namespace ib

struct IbetaCF {
  double K, Kp, Kq;
};

// K = 1 + d_1/(1 + d_2/(1 + ...)) for I_y(p, q), with
//   d_(2m+1) = -(p+m)(p+q+m) y / ((p+2m)(p+2m+1)),
//   d_(2m)   = m(q-m) y / ((p+2m-1)(p+2m)),
// and (DERIVS) ∂K/∂p, ∂K/∂q.  sp and sq are the sizes of the other terms
// beside K_p/K and K_q/K in ∂ ln J: the derivatives are converged once
// their change is below rounding of that sum.
template <bool DERIVS>
__device__ inline IbetaCF ibeta_cf(double p, double q, double y, double sp, double sq) {
  // A_(n-1), A_(n-2), B_(n-1), B_(n-2) and their p- and q-derivatives.
  double A1 = 1.0, A2 = 1.0, B1 = 1.0, B2 = 0.0;
  double Ap1 = 0.0, Ap2 = 0.0, Bp1 = 0.0, Bp2 = 0.0;
  double Aq1 = 0.0, Aq2 = 0.0, Bq1 = 0.0, Bq2 = 0.0;
  double K = 1.0, Kp = 0.0, Kq = 0.0;
  const double pq = p + q;
  auto step = [&](double d, double dp, double dq) {
    const double A = fma(d, A2, A1), B = fma(d, B2, B1);
    if (DERIVS) {
      const double Ap = fma(d, Ap2, fma(dp, A2, Ap1)), Bp = fma(d, Bp2, fma(dp, B2, Bp1));
      const double Aq = fma(d, Aq2, fma(dq, A2, Aq1)), Bq = fma(d, Bq2, fma(dq, B2, Bq1));
      Ap2 = Ap1, Bp2 = Bp1, Aq2 = Aq1, Bq2 = Bq1;
      Ap1 = Ap, Bp1 = Bp, Aq1 = Aq, Bq1 = Bq;
    }
    A2 = A1, B2 = B1, A1 = A, B1 = B;
  };
  // The d_n and their p- and q-derivatives share reciprocals (two for an
  // odd term, one for an even one; products kept apart so that no
  // intermediate overflows before the parameters do), and the recurrences
  // are rescaled by 1/B_n once per pair of terms, after which B_n = 1 and
  // K = A_n.  Two terms grow the recurrences by at most (1 + |d|)^2 with
  // |d| below about (p + q) / p, inside the exponent range for parameters
  // below 1e150.
  {  // counted loop: reaching the cap is recorded (note_unconverged)
    int m = 0;
    for (; m < ib::kMaxPairs; ++m) {
      const double md = m;
      {  // d_(2m+1) = -u v y / (w w1); ∂p ln d = 1/u + 1/v - 1/w - 1/w1, ∂q ln d = 1/v
        const double u = p + md, v = pq + md, w = p + 2.0 * md, w1 = w + 1.0;
        const double uv = u * v, ww = w * w1;
        if (DERIVS) {
          const double ruv = 1.0 / uv, rww = 1.0 / ww;
          const double d = -(uv * y) * rww;
          step(d, d * ((u + v) * ruv - (w + w1) * rww), d * (u * ruv));
        } else {
          step(-(uv * y) / ww, 0.0, 0.0);
        }
      }
      {  // d_(2m+2) = (q - k) k y / (w w1); ∂p ln d = -1/w - 1/w1, ∂q d = k y / (w w1)
        const double k = md + 1.0, w = p + 2.0 * md + 1.0, w1 = w + 1.0;
        const double rho = 1.0 / (w * w1);
        const double r = k * y * rho;
        const double d = (q - k) * r;
        step(d, DERIVS ? -d * ((w + w1) * rho) : 0.0, r);
      }
      const double s = 1.0 / (fabs(B1) > 1e-300 ? B1 : 1e-300);
      A1 *= s, A2 *= s, B2 *= s;
      B1 = 1.0;
      if (DERIVS) Ap1 *= s, Ap2 *= s, Bp1 *= s, Bp2 *= s, Aq1 *= s, Aq2 *= s, Bq1 *= s, Bq2 *= s;
      const double Kn = A1;
      bool done = fabs(Kn - K) <= ib::kTol * fabs(Kn);
      if (DERIVS) {
        const double Kpn = fma(-Kn, Bp1, Ap1), Kqn = fma(-Kn, Bq1, Aq1);
        done = done && fabs(Kpn - Kp) <= ib::kTolD * (fabs(Kpn) + fabs(Kn) * sp) &&
               fabs(Kqn - Kq) <= ib::kTolD * (fabs(Kqn) + fabs(Kn) * sq);
        Kp = Kpn, Kq = Kqn;
      }
      K = Kn;
      if (done) break;
    }
    if (m >= ib::kMaxPairs) note_unconverged();
  }
  return {K, Kp, Kq};
}

// I_x(a, b) and (DERIVS) its first derivatives, for 0 < x < 1 and finite
// a, b > 0.  Without DERIVS only v is formed, with the reference's closed
// forms at a = 1 or b = 1; with DERIVS v is not formed.
template <bool DERIVS>
__device__ inline IbetaOut ibeta_eval(double x, double a, double b) {
  IbetaOut r{0.0, 0.0, 0.0, 0.0};
  const double lx = log(x), l1x = log1p(-x);
  if (!DERIVS) {
    if (a == 1.0 && b == 1.0) return r.v = x, r;
    if (a == 1.0) return r.v = -expm1(b * l1x), r;
    if (b == 1.0) return r.v = exp(a * lx), r;
  }
  const bool swap = x > (a + 1.0) / (a + b + 2.0);
  const double p = swap ? b : a, q = swap ? a : b;
  const double y = swap ? 1.0 - x : x, ly = swap ? l1x : lx, l1y = swap ? lx : l1x;
  const double lnB = log_beta_pos(p, q);
  double pdp = 0.0, pdq = 0.0;
  if (DERIVS) pdp = psi_diff(p, q), pdq = psi_diff(q, p);
  const IbetaCF cf = ibeta_cf<DERIVS>(p, q, y, fabs(ly) + fabs(pdp) + 1.0 / p, fabs(l1y) + fabs(pdq));
  const double J = exp(((p * ly + q * l1y) - lnB) - log(p)) / cf.K;
  if (!DERIVS) {
    r.v = swap ? 1.0 - J : J;
    return r;
  }
  const double Jp = J * (((ly - pdp) - 1.0 / p) - cf.Kp / cf.K);
  const double Jq = J * ((l1y - pdq) - cf.Kq / cf.K);
  r.da = swap ? -Jq : Jp;
  r.db = swap ? -Jp : Jq;
  r.dx = exp(((a - 1.0) * lx + (b - 1.0) * l1x) - lnB);
  return r;
}

// Out of line: the double backward evaluates the derivatives at five points,
// and one copy of the fraction keeps the loop resident in the instruction
// cache.
static __device__ __noinline__ IbetaOut ibeta_derivs(double x, double a, double b) {
  return ibeta_eval<true>(x, a, b);
}

__device__ __forceinline__ bool ibeta_params_ok(double a, double b) {
  return a > 0.0 && b > 0.0 && isfinite(a) && isfinite(b);
}

// Region of (x, a, b) by the expected length of the continued fraction, so
// that the map kernel gives each warp lanes of similar cost: the fraction
// takes longer the larger the smaller parameter (bucketed by its binary
// logarithm, 0 .. 6) and the closer x lies to the swap point
// (a+1)/(a+b+2), within three standard deviations of the beta distribution
// or not.  The closed forms (a = 1 or b = 1) and the points outside the
// domain are regions of their own.  Numbered by decreasing cost.
constexpr int kIbRegions = 16;
__device__ __forceinline__ int ibeta_classify(double xd, double ad, double bd) {
  if (!(xd > 0.0 && xd < 1.0) || !ibeta_params_ok(ad, bd)) return kIbRegions - 1;
  if (ad == 1.0 || bd == 1.0) return kIbRegions - 2;
  const float x = (float)xd, a = (float)ad, b = (float)bd;
  const int lb = min(6, (int)__log2f(1.0f + fminf(a, b)));
  const float s = a + b, xs = (a + 1.0f) / (s + 2.0f);
  const float sd = sqrtf(a * b / (s * s * (s + 1.0f)));
  const bool near = fabsf(x - xs) < 3.0f * sd;
  return (6 - lb) * 2 + (near ? 0 : 1);
}

template <typename T_>
struct IbetaFwd {  // in = {x, a, b}
  using T = T_;
  static constexpr int NIN = 3, NOUT = 1, R = kIbRegions;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) { return ibeta_classify(in[0], in[1], in[2]); }
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double x = in[0], a = in[1], b = in[2];
    double v;
    if (isnan(x) || !ibeta_params_ok(a, b))
      v = CUDART_NAN;
    else if (x <= 0.0)
      v = 0.0;
    else if (x >= 1.0)
      v = 1.0;
    else
      v = ibeta_eval<false>(x, a, b).v;
    out[0] = (T)v;
  }
};

template <typename T_>
struct IbetaBwd {  // in = {grad, x, a, b}, out = {grad_x, grad_a, grad_b}
  using T = T_;
  static constexpr int NIN = 4, NOUT = 3, R = kIbRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) { return ibeta_classify(in[1], in[2], in[3]); }
  __device__ static void eval(int, const T* in, T* out, uint32_t mask) {
    const double g = in[0], x = in[1], a = in[2], b = in[3];
    double gx = 0.0, ga = 0.0, gb = 0.0;
    if (x <= 0.0 || x >= 1.0) {
    } else if (isnan(x) || !ibeta_params_ok(a, b)) {
      gx = ga = gb = CUDART_NAN;
    } else if (!(mask & 6u)) {  // only ∂x: the density, no fraction
      gx = g * exp(((a - 1.0) * log(x) + (b - 1.0) * log1p(-x)) - log_beta_pos(a, b));
    } else {
      const IbetaOut d = ibeta_derivs(x, a, b);
      gx = g * d.dx, ga = g * d.da, gb = g * d.db;
    }
    out[0] = (mask & 1u) ? (T)gx : T(0);
    out[1] = (mask & 2u) ? (T)ga : T(0);
    out[2] = (mask & 4u) ? (T)gb : T(0);
  }
};

template <typename T_>
struct IbetaBwdBwd {  // in = {gg_x, gg_a, gg_b, grad, x, a, b}, out = {grad_grad_output, grad_x, grad_a, grad_b}
  using T = T_;
  static constexpr int NIN = 7, NOUT = 4, R = kIbRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) { return ibeta_classify(in[4], in[5], in[6]); }
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double ggx = in[0], gga = in[1], ggb = in[2], g = in[3], x = in[4], a = in[5], b = in[6];
    if (x <= 0.0 || x >= 1.0) {
      out[0] = out[1] = out[2] = out[3] = T(0);
      return;
    }
    if (isnan(x) || !ibeta_params_ok(a, b)) {
      out[0] = out[1] = out[2] = out[3] = (T)CUDART_NAN;
      return;
    }
    const IbetaOut d = ibeta_derivs(x, a, b);
    const double lx = log(x), l1x = log1p(-x);
    const double hxx = d.dx * ((a - 1.0) / x - (b - 1.0) / (1.0 - x));
    const double hxa = d.dx * (lx - psi_diff(a, b));
    const double hxb = d.dx * (l1x - psi_diff(b, a));
    // Central differences of the analytic ∂a, ∂b (the points' own spacing
    // is the divisor).
    const double ap = a * (1.0 + ib::kStep), am = a * (1.0 - ib::kStep);
    const double bp = b * (1.0 + ib::kStep), bm = b * (1.0 - ib::kStep);
    const IbetaOut dap = ibeta_derivs(x, ap, b), dam = ibeta_derivs(x, am, b);
    const IbetaOut dbp = ibeta_derivs(x, a, bp), dbm = ibeta_derivs(x, a, bm);
    const double haa = (dap.da - dam.da) / (ap - am);
    const double hbb = (dbp.db - dbm.db) / (bp - bm);
    const double hab = 0.5 * ((dap.db - dam.db) / (ap - am) + (dbp.da - dbm.da) / (bp - bm));
    out[0] = (T)(ggx * d.dx + gga * d.da + ggb * d.db);
    out[1] = (T)(g * (ggx * hxx + gga * hxa + ggb * hxb));
    out[2] = (T)(g * (ggx * hxa + gga * haa + ggb * hab));
    out[3] = (T)(g * (ggx * hxb + gga * hab + ggb * hbb));
  }
};

}  // namespace tsb
