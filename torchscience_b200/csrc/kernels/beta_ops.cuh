// log_beta, beta and polygamma: functors of the forward, backward and
// double-backward entry points (reference: log_beta.h:10-13,
// log_beta_backward.h:10-17, log_beta_backward_backward.h:10-33,
// beta.h:12-15, beta_backward.h:13-27, beta_backward_backward.h:10-30,
// polygamma.h:45-62, polygamma_backward.h:10-19,
// polygamma_backward_backward.h:10-22).  Every argument costs about the same
// (no region split); float data is evaluated in FP64 and rounded once.
#pragma once

#include "beta_math.cuh"
#include "dispatch.cuh"

namespace tsb {

// Second-order pieces of ln B: ∂a, ∂b, ∂aa, ∂bb, ∂ab.
struct LogBetaDerivs {
  double da, db, daa, dbb, dab;
};
__device__ inline LogBetaDerivs log_beta_derivs(double a, double b) {
  return {log_beta_da(a, b), log_beta_da(b, a), log_beta_daa(a, b), log_beta_daa(b, a), -trigamma_d(a + b)};
}

template <typename T_>
struct LogBetaFwd {
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) { out[0] = (T)log_beta_d(in[0], in[1]); }
};

template <typename T_>
struct LogBetaBwd {  // in = {grad, a, b}, out = {grad_a, grad_b}
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = 1;
  static constexpr bool REDUCE = true;
  __device__ static void eval(int, const T* in, T* out, uint32_t mask) {
    const double g = in[0], a = in[1], b = in[2];
    out[0] = (mask & 1u) ? (T)(g * log_beta_da(a, b)) : T(0);
    out[1] = (mask & 2u) ? (T)(g * log_beta_da(b, a)) : T(0);
  }
};

template <typename T_>
struct LogBetaBwdBwd {  // in = {gg_a, gg_b, grad, a, b}, out = {grad_grad_output, grad_a, grad_b}
  using T = T_;
  static constexpr int NIN = 5, NOUT = 3, R = 1;
  static constexpr bool REDUCE = true;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double gga = in[0], ggb = in[1], g = in[2];
    const LogBetaDerivs d = log_beta_derivs(in[3], in[4]);
    out[0] = (T)(gga * d.da + ggb * d.db);
    out[1] = (T)(g * (gga * d.daa + ggb * d.dab));
    out[2] = (T)(g * (gga * d.dab + ggb * d.dbb));
  }
};

template <typename T_>
struct BetaFwd {
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) { out[0] = (T)beta_d(in[0], in[1]); }
};

template <typename T_>
struct BetaBwd {  // in = {grad, a, b}: ∂B/∂a = B (ψ(a) - ψ(a+b))
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = 1;
  static constexpr bool REDUCE = true;
  __device__ static void eval(int, const T* in, T* out, uint32_t mask) {
    const double g = in[0], a = in[1], b = in[2], gB = g * beta_d(a, b);
    out[0] = (mask & 1u) ? (T)(gB * log_beta_da(a, b)) : T(0);
    out[1] = (mask & 2u) ? (T)(gB * log_beta_da(b, a)) : T(0);
  }
};

template <typename T_>
struct BetaBwdBwd {  // ∂²B = B (∂ ln B ∂ ln B + ∂² ln B)
  using T = T_;
  static constexpr int NIN = 5, NOUT = 3, R = 1;
  static constexpr bool REDUCE = true;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double gga = in[0], ggb = in[1], g = in[2], a = in[3], b = in[4];
    const double B = beta_d(a, b);
    const LogBetaDerivs d = log_beta_derivs(a, b);
    const double haa = B * fma(d.da, d.da, d.daa), hab = B * fma(d.da, d.db, d.dab), hbb = B * fma(d.db, d.db, d.dbb);
    out[0] = (T)(B * (gga * d.da + ggb * d.db));
    out[1] = (T)(g * (gga * haa + ggb * hab));
    out[2] = (T)(g * (gga * hab + ggb * hbb));
  }
};

// Region of an order: n = 0 .. 3 take their own evaluators (regions 0 .. 3),
// higher orders the Hurwitz zeta, whose direct-term count grows with n
// (buckets of 4 orders up to n = 43, then one more); z < 0 adds the
// reflection's second sum (its own bucket).  Regions are numbered by
// decreasing cost.
constexpr int kPgRegions = 16;
__device__ __forceinline__ int polygamma_classify(int n, double z) {
  if (n < 0 || isnan(z)) return kPgRegions - 1;
  if (z < 0.0) return 0;
  if (n <= 3) return kPgRegions - 2 - n;  // 14 .. 11
  const int b = (n - 4) >> 2;               // 0 .. 9 for n < 44
  return b >= 9 ? 1 : 10 - b;               // 10 .. 2, and 1 for n >= 40
}

template <typename T_>
struct PolygammaFwd {  // in = {n, z}
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = kPgRegions;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) { return polygamma_classify(polygamma_order(in[0]), in[1]); }
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    out[0] = (T)polygamma_d(polygamma_order(in[0]), in[1]);
  }
};

template <typename T_>
struct PolygammaBwd {  // in = {grad, n, z}, out = {grad_n = 0, grad_z = grad·ψ^(n+1)(z)}
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = kPgRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) {
    return polygamma_classify(polygamma_order((double)in[1] + 1.0), in[2]);
  }
  __device__ static void eval(int, const T* in, T* out, uint32_t mask) {
    out[0] = T(0);
    out[1] = (mask & 2u) ? (T)((double)in[0] * polygamma_d(polygamma_order((double)in[1] + 1.0), in[2])) : T(0);
  }
};

template <typename T_>
struct PolygammaBwdBwd {  // in = {gg_n, gg_z, grad, n, z}
  using T = T_;
  static constexpr int NIN = 5, NOUT = 3, R = kPgRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) {
    return polygamma_classify(polygamma_order((double)in[3] + 2.0), in[4]);
  }
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double ggz = in[1], g = in[2], n = in[3], z = in[4];
    out[0] = (T)(ggz * polygamma_d(polygamma_order(n + 1.0), z));
    out[1] = T(0);
    out[2] = (T)(ggz * g * polygamma_d(polygamma_order(n + 2.0), z));
  }
};

}  // namespace tsb

// ------------------------------------------------------------ complex data
// log_beta and beta of complex64 / complex128 arguments (evaluated in
// complex128): ln B(a, b) = lnΓ(a) + lnΓ(b) - lnΓ(a+b) with the principal
// lnΓ (log_beta.h:15-17 takes the same sum of its complex log_gamma), and
// B = exp(ln B) (beta.h:13-15).  Gradients follow the gamma family's
// convention (PyTorch's conjugate Wirtinger gradients): for f(a, b)
// holomorphic in each argument, backward = (g·conj(f_a), g·conj(f_b)) and the
// double backward = (gg_a·f_a + gg_b·f_b,
//   conj(gg_a)·g·conj(f_aa) + conj(gg_b)·g·conj(f_ab),
//   conj(gg_a)·g·conj(f_ab) + conj(gg_b)·g·conj(f_bb)),
// with f_a = ψ(a) - ψ(a+b), f_aa = ψ'(a) - ψ'(a+b), f_ab = -ψ'(a+b) for
// ln B, and B times the logarithmic derivatives for B.  (The reference's
// complex log_beta_backward.h:19-27 does not conjugate.)
#include "complex_gamma.cuh"

namespace tsb {

struct CBetaDerivs {
  cdouble f, fa, fb, faa, fab, fbb;
};
template <bool EXP, int ORDER>
__device__ inline CBetaDerivs cbeta_derivs(cdouble a, cdouble b) {
  CBetaDerivs d;
  const cdouble s = a + b;
  const cdouble lb = loggamma_c(a) + loggamma_c(b) - loggamma_c(s);
  d.f = EXP ? cuda::std::exp(lb) : lb;
  d.fa = d.fb = d.faa = d.fab = d.fbb = cdouble(0.0, 0.0);
  if (ORDER >= 1) {
    const cdouble ps = digamma_c(s), da = digamma_c(a) - ps, db = digamma_c(b) - ps;
    d.fa = EXP ? d.f * da : da;
    d.fb = EXP ? d.f * db : db;
    if (ORDER >= 2) {
      const cdouble p1 = trigamma_c(s), daa = trigamma_c(a) - p1, dbb = trigamma_c(b) - p1, dab = -p1;
      d.faa = EXP ? d.f * (da * da + daa) : daa;
      d.fab = EXP ? d.f * (da * db + dab) : dab;
      d.fbb = EXP ? d.f * (db * db + dbb) : dbb;
    }
  }
  return d;
}

template <bool EXP>
struct CBetaFwd {  // in = {a, b}
  using T = cdouble;
  static constexpr int NIN = 2, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) { out[0] = cbeta_derivs<EXP, 0>(in[0], in[1]).f; }
};
template <bool EXP>
struct CBetaBwd {  // in = {grad, a, b}, out = {grad_a, grad_b}
  using T = cdouble;
  static constexpr int NIN = 3, NOUT = 2, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const CBetaDerivs d = cbeta_derivs<EXP, 1>(in[1], in[2]);
    out[0] = in[0] * cuda::std::conj(d.fa);
    out[1] = in[0] * cuda::std::conj(d.fb);
  }
};
template <bool EXP>
struct CBetaBwdBwd {  // in = {gg_a, gg_b, grad, a, b}, out = {grad_grad_output, grad_a, grad_b}
  using T = cdouble;
  static constexpr int NIN = 5, NOUT = 3, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const cdouble gga = in[0], ggb = in[1], g = in[2];
    const CBetaDerivs d = cbeta_derivs<EXP, 2>(in[3], in[4]);
    const cdouble cga = cuda::std::conj(gga), cgb = cuda::std::conj(ggb);
    out[0] = gga * d.fa + ggb * d.fb;
    out[1] = g * (cga * cuda::std::conj(d.faa) + cgb * cuda::std::conj(d.fab));
    out[2] = g * (cga * cuda::std::conj(d.fab) + cgb * cuda::std::conj(d.fbb));
  }
};

}  // namespace tsb
