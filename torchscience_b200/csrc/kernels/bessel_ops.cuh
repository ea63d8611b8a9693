// Bessel J_ν, Y_ν, I_ν, K_ν of real order and J_0: functors of the forward,
// backward (grad_n, grad_z) and double-backward entry points, with the
// reference's conventions for x <= 0, integer and negative orders
// (bessel_j.h:240-316, bessel_y.h:131-193, modified_bessel_i.h:271-366,
// modified_bessel_k.h:249-307, bessel_j_0.h:91-129).
//
// ∂/∂x comes with each evaluation; ∂²/∂x² from Bessel's equation.  ∂/∂ν
// has no practical closed form for real order (the reference also uses
// central differences, bessel_j_backward.h:17-28); here it is a central
// difference of the accurate FP64 evaluator with step ε^(1/3)·max(1, |ν|)
// (ε^(1/4) for the second derivative), only computed when grad_n is
// requested.
#pragma once

#include <type_traits>

#include "bessel_math.cuh"
#include "dispatch.cuh"

namespace tsb {

enum BesselKind : int { kBJ = 0, kBY = 1, kBI = 2, kBK = 3 };
enum BesselRegion : int { kBsSpecial = 0, kBsSeries = 1, kBsMid = 2, kBsLarge = 3, kBsJ01 = 4, kBsRegions = 5 };

// J at order 0 or ±1 with finite, non-zero x: the dedicated J0/J1 path.
__device__ __forceinline__ bool bessel_j01_order(double nu) { return nu == 0.0 || fabs(nu) == 1.0; }

// Evaluation region (also the unit of compaction).  Mixed kernels run
// kBsSeries (x < 2, order >= 0 or integer) in FP32 and the others in FP64;
// kBsJ01 is J at order 0, ±1.
template <int KIND>
__device__ __forceinline__ int bessel_classify(double nu, double x) {
  if (isnan(nu) || isnan(x) || isinf(nu) || isinf(x) || x == 0.0) return kBsSpecial;
  if (KIND == kBJ && bessel_j01_order(nu)) return kBsJ01;
  if ((KIND == kBY || KIND == kBK) && x < 0.0) return kBsSpecial;
  const double ax = fabs(x), an = fabs(nu);
  if (ax < 2.0) return (nu >= 0.0 || an == floor(an)) ? kBsSeries : kBsMid;
  if (ax >= 25.0 && (KIND == kBI || KIND == kBK || an < ax)) return kBsLarge;
  return kBsMid;
}

template <typename T>
struct BV {
  T v, d;  // value, d/dx
};

__device__ __forceinline__ bool odd_integer(double a) { return fmod(a, 2.0) == 1.0; }
__device__ __forceinline__ bool odd_integer(float a) { return fmodf(a, 2.0f) == 1.0f; }

// J_ν(0) / I_ν(0) per the reference (bessel_j.h:253-266, modified_bessel_i.h:278-288).
template <typename T>
__device__ __forceinline__ T bessel_at_zero(T nu) {
  if (nu == T(0)) return T(1);
  if (nu > T(0)) return T(0);
  if (nu == floor(nu)) return T(0);
  return T(CUDART_INF);
}

template <typename T, int KIND>
__device__ inline BV<T> bessel_eval(T nu, T x) {
  const T nan = T(CUDART_NAN), inf = T(CUDART_INF);
  if (isnan(nu) || isnan(x) || isinf(nu)) return {nan, nan};
  if (KIND == kBY || KIND == kBK) {
    if (x < T(0)) return {nan, nan};
    if (x == T(0)) return KIND == kBY ? BV<T>{-inf, inf} : BV<T>{inf, -inf};
    if (isinf(x)) return {T(0), T(0)};
  }
  const T an = fabs(nu);
  const bool is_int = an == floor(an);
  if (x == T(0)) {  // J, I: derivative as (C_{ν-1}(0) ∓ C_{ν+1}(0))/2, like the reference's backward
    const T c0 = bessel_at_zero(nu), cm = bessel_at_zero(nu - T(1)), cp = bessel_at_zero(nu + T(1));
    return {c0, KIND == kBJ ? T(0.5) * (cm - cp) : T(0.5) * (cm + cp)};
  }
  if (isinf(x)) {
    if (KIND == kBJ) return {T(0), T(0)};
    if (x > T(0)) return {inf, inf};
    if (!is_int) return {nan, nan};
    const T s = odd_integer(an) ? T(-1) : T(1);
    return {s * inf, -s * inf};
  }
  if (KIND == kBJ && bessel_j01_order((double)nu)) {  // J0' = -J1, J1' = J0 - J1/x, J_{-1} = -J_1
    const J01 b = bessel_j01_call((double)x);
    if (nu == T(0)) return {(T)b.j0, (T)(-b.j1)};
    const double v = b.j1, d = b.j0 - b.j1 / (double)x;
    return nu > T(0) ? BV<T>{(T)v, (T)d} : BV<T>{(T)(-v), (T)(-d)};
  }
  const T ax = fabs(x);
  T v, d;
  if (KIND == kBJ || KIND == kBY) {
    const bool need_y = KIND == kBY || (nu < T(0) && !is_int);
    const bool need_j = KIND == kBJ || (nu < T(0) && !is_int);  // Y_{-a} takes J_a (DLMF 10.4.7)
    const JY<T> r = !need_y ? besseljy_pos<T, false>(an, ax)
                            : (need_j ? besseljy_pos<T, true>(an, ax) : besseljy_pos<T, true, false>(an, ax));
    if (nu >= T(0) || is_int) {
      v = KIND == kBJ ? r.j : r.y;
      d = KIND == kBJ ? r.jp : r.yp;
      if (nu < T(0) && odd_integer(an)) {  // C_{-n} = (-1)^n C_n
        v = -v;
        d = -d;
      }
    } else {  // DLMF 10.4.7: J_{-a} = cos(aπ)J_a - sin(aπ)Y_a, Y_{-a} = sin(aπ)J_a + cos(aπ)Y_a
      T s, c;
      bx::sincospi_(an, &s, &c);
      if (KIND == kBJ) {
        v = c * r.j - s * r.y;
        d = c * r.jp - s * r.yp;
      } else {
        v = s * r.j + c * r.y;
        d = s * r.jp + c * r.yp;
      }
    }
  } else {
    bool scaled = false;
    const bool need_k = KIND == kBK || (nu < T(0) && !is_int);
    const IK<T> r = KIND == kBK ? besselik_pos<T, false, true>(an, ax, scaled)
                                : (need_k ? besselik_pos<T, true, true>(an, ax, scaled)
                                          : besselik_pos<T, true, false>(an, ax, scaled));
    T i = r.i, ip = r.ip, k = r.k, kp = r.kp;
    if (scaled) {  // undo e^{-x} I, e^{x} K (split e^x so I does not overflow early)
      const T eh = bx::exp_(T(0.5) * ax), em = bx::exp_(-ax);
      i = (i * eh) * eh;
      ip = (ip * eh) * eh;
      k *= em;
      kp *= em;
    }
    if (KIND == kBK) {
      v = k;
      d = kp;
    } else if (nu >= T(0) || is_int) {
      v = i;
      d = ip;
    } else {  // DLMF 10.27.2: I_{-a} = I_a + (2/π) sin(aπ) K_a
      T s, c;
      bx::sincospi_(an, &s, &c);
      const T f = T(2) / T(CUDART_PI) * s;
      v = i + f * k;
      d = ip + f * kp;
    }
  }
  if (x < T(0)) {  // J, I only: reference sign conventions for negative x
    T f;
    if (is_int) {
      f = odd_integer(an) ? T(-1) : T(1);
    } else {
      T s;
      bx::sincospi_(nu, &s, &f);
    }
    v *= f;
    d = -f * d;
  }
  return {v, d};
}

// Second x-derivative from Bessel's equation (J, Y) or the modified one (I, K).
template <typename T, int KIND>
__device__ __forceinline__ T bessel_d2(T nu, T x, const BV<T>& b) {
  const T r = nu / x;
  if (KIND == kBJ || KIND == kBY) return -b.d / x - (T(1) - r * r) * b.v;
  return -b.d / x + (T(1) + r * r) * b.v;
}

// ν-derivatives by central differences of the FP64 evaluator.
struct BesselNuDerivs {
  double dv, dd;  // ∂v/∂ν, ∂(dv/dx)/∂ν
  double dvv;     // ∂²v/∂ν²
};
template <int KIND, bool SECOND>
__device__ inline BesselNuDerivs bessel_nu_derivs(double nu, double x, const BV<double>& b0) {
  BesselNuDerivs o;
  const double h = 6.0554544523933395e-06 * fmax(1.0, fabs(nu));  // ε^(1/3)
  const BV<double> bp = bessel_eval<double, KIND>(nu + h, x), bm = bessel_eval<double, KIND>(nu - h, x);
  o.dv = (bp.v - bm.v) / (2.0 * h);
  o.dd = (bp.d - bm.d) / (2.0 * h);
  o.dvv = 0.0;
  if (SECOND) {
    const double h2 = 1.2207031250e-04 * fmax(1.0, fabs(nu));  // ε^(1/4)
    const BV<double> cp = bessel_eval<double, KIND>(nu + h2, x), cm = bessel_eval<double, KIND>(nu - h2, x);
    o.dvv = (cp.v - 2.0 * b0.v + cm.v) / (h2 * h2);
  }
  return o;
}

// Value (+ d/dx) in the mixed kernels: FP32 in the kBsSeries region (J, I, K;
// Y's series region is Temme's series in FP64 either way); for K (no zeros)
// also in the Steed (Temme's CF2) and Hankel regions, with the order
// recurrences in FP64; FP64 otherwise.  Measured against the FP64 kernels on
// configuration-3 points, Steed's CF1 for J, Y and I carries up to ~2e-5 in
// FP32 and I's Hankel path up to 1.2e-6, so those stay FP64 (J and Y take
// FP32 in the Hankel region through bessel_first below).  Non-finite FP32
// results (values at the edge of FP32 range) are redone in FP64.
template <typename T, int KIND>
__device__ __forceinline__ BV<T> bessel_value(int region, T nu, T x) {
  if constexpr (std::is_same<T, float>::value) {
    const bool fp32 = (region == kBsSeries && KIND != kBY) || (KIND == kBK && (region == kBsMid || region == kBsLarge));
    if (fp32) {
      const BV<float> f = bessel_eval<float, KIND>(nu, x);
      if (isfinite(f.v) && isfinite(f.d)) return f;
    }
    const BV<double> dd = bessel_eval<double, KIND>((double)nu, (double)x);
    return {(float)dd.v, (float)dd.d};
  } else {
    return bessel_eval<double, KIND>(nu, x);
  }
}

// J and Y in the mixed kernels' Hankel region (x >= 25, ν < x): FP32, with
// the elements next to a zero of the requested quantity declined to the FP64
// evaluator (the map kernel's rescue list).  Near a zero the FP32 result keeps
// its absolute accuracy, about 3 ulp of the local modulus M, but not its
// relative accuracy.  With the Debye phase rate w = sqrt(1 - (ν/x)²) the
// modulus is M² ≈ C² + (C'/w)²; an FP32 value is kept when |C| >= 0.3 M, a
// derivative when |C'| >= 0.3 w M, which bounds their relative error by
// about 3·6e-8 / 0.3 = 6e-7.  For x <= ν neither function has a zero.
constexpr float kBsKeep = 0.3f;
__device__ __forceinline__ bool bessel_fp32_kept(float nu, float x, float v, float d, bool deriv) {
  if (!isfinite(v) || !isfinite(d)) return false;
  const float r = fabsf(nu) / x;
  if (r >= 1.0f) return true;
  const float w2 = 1.0f - r * r;
  const float m2 = v * v + d * d / w2;
  if (!isfinite(m2)) return false;
  return deriv ? d * d >= kBsKeep * kBsKeep * w2 * m2 : v * v >= kBsKeep * kBsKeep * m2;
}
template <typename T, int KIND>
__device__ __forceinline__ bool bessel_first(int region, T nu, T x, bool deriv, BV<T>& out) {
  if constexpr (std::is_same<T, float>::value && (KIND == kBJ || KIND == kBY)) {
    if (region == kBsLarge && nu >= 0.0f && x > 0.0f) {
      const BV<float> f = bessel_eval<float, KIND>(nu, x);
      if (!bessel_fp32_kept(nu, x, f.v, f.d, deriv)) return false;
      out = f;
      return true;
    }
  }
  out = bessel_value<T, KIND>(region, nu, x);
  return true;
}
template <typename T, int KIND>
__device__ __forceinline__ BV<T> bessel_rescue(T nu, T x) {
  const BV<double> dd = bessel_eval<double, KIND>((double)nu, (double)x);
  return {(T)dd.v, (T)dd.d};
}

template <int KIND, typename T_>
struct BesselFwd {
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = kBsRegions;
  static constexpr bool REDUCE = false;
  static constexpr bool RESCUE = std::is_same<T, float>::value && (KIND == kBJ || KIND == kBY);
  __device__ static int classify(const T* in) { return bessel_classify<KIND>((double)in[0], (double)in[1]); }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) { out[0] = bessel_value<T, KIND>(r, in[0], in[1]).v; }
  __device__ static bool eval_first(int r, const T* in, T* out, uint32_t) {
    BV<T> b;
    if (!bessel_first<T, KIND>(r, in[0], in[1], false, b)) return false;
    out[0] = b.v;
    return true;
  }
  __device__ static void eval_rescue(int, const T* in, T* out, uint32_t) { out[0] = bessel_rescue<T, KIND>(in[0], in[1]).v; }
};

// in = {grad, n, z}, out = {grad_n, grad_z}
template <int KIND, typename T_>
struct BesselBwd {
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = kBsRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) { return bessel_classify<KIND>((double)in[1], (double)in[2]); }
  __device__ static void eval(int r, const T* in, T* out, uint32_t mask) {
    if (mask & 1u) {  // grad_n needs the FP64 central difference
      const double nu = in[1], x = in[2], g = in[0];
      const BV<double> b = bessel_eval<double, KIND>(nu, x);
      const BesselNuDerivs dn = bessel_nu_derivs<KIND, false>(nu, x, b);
      out[0] = (T)(g * dn.dv);
      out[1] = (T)(g * b.d);
      return;
    }
    out[0] = T(0);
    out[1] = in[0] * bessel_value<T, KIND>(r, in[1], in[2]).d;
  }
  static constexpr bool RESCUE = std::is_same<T, float>::value && (KIND == kBJ || KIND == kBY);
  __device__ static bool eval_first(int r, const T* in, T* out, uint32_t mask) {
    if (mask & 1u) {
      eval(r, in, out, mask);
      return true;
    }
    BV<T> b;
    if (!bessel_first<T, KIND>(r, in[1], in[2], true, b)) return false;
    out[0] = T(0);
    out[1] = in[0] * b.d;
    return true;
  }
  __device__ static void eval_rescue(int, const T* in, T* out, uint32_t) {
    out[0] = T(0);
    out[1] = in[0] * bessel_rescue<T, KIND>(in[1], in[2]).d;
  }
};

// in = {gg_n, gg_z, grad, n, z}, out = {grad_grad_output, grad_n, grad_z}
template <int KIND, typename T_>
struct BesselBwdBwd {
  using T = T_;
  static constexpr int NIN = 5, NOUT = 3, R = kBsRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) { return bessel_classify<KIND>((double)in[3], (double)in[4]); }
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double ggn = in[0], ggz = in[1], g = in[2], nu = in[3], x = in[4];
    const BV<double> b = bessel_eval<double, KIND>(nu, x);
    const BesselNuDerivs dn = bessel_nu_derivs<KIND, true>(nu, x, b);
    const double d2 = bessel_d2<double, KIND>(nu, x, b);
    out[0] = (T)(ggn * dn.dv + ggz * b.d);
    out[1] = (T)(g * (ggn * dn.dvv + ggz * dn.dd));
    out[2] = (T)(g * (ggn * dn.dd + ggz * d2));
  }
};

// J_0 (bessel_j_0): the order-0/1 path with no region split (every finite
// argument costs about the same); J0(0) = 1, J0(±inf) = 0 as in the
// reference (bessel_j_0.h:91-129).  Float data is evaluated in FP64 and
// rounded once.
template <typename T_>
struct BesselJ0Fwd {
  using T = T_;
  static constexpr int NIN = 1, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double x = in[0];
    double v;
    if (isnan(x)) v = x;
    else if (isinf(x)) v = 0.0;
    else if (x == 0.0) v = 1.0;
    else v = bessel_j01<true, false>(x).j0;
    out[0] = (T)v;
  }
};
template <typename T_>
struct BesselJ0Bwd {  // in = {grad, z}: grad * J0'(z) = -grad * J1(z)
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double g = in[0], x = in[1];
    double d;
    if (isnan(x)) d = x;
    else if (isinf(x)) d = 0.0;
    else d = -bessel_j01<false, true>(x).j1;
    out[0] = (T)(g * d);
  }
};
template <typename T_>
struct BesselJ0BwdBwd {  // in = {gg, grad, z}: {gg·J0'(z), gg·grad·J0''(z)}, J0'' = J1/z - J0
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = 1;
  static constexpr bool REDUCE = true;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double gg = in[0], g = in[1], x = in[2];
    double d1, d2;
    if (isnan(x)) {
      d1 = d2 = x;
    } else if (isinf(x)) {
      d1 = d2 = 0.0;
    } else if (x == 0.0) {
      d1 = 0.0;
      d2 = -0.5;
    } else {
      const J01 b = bessel_j01<true, true, TSB_B01_UNROLL>(x);
      d1 = -b.j1;
      d2 = b.j1 / x - b.j0;
    }
    out[0] = (T)(gg * d1);
    out[1] = (T)(gg * g * d2);
  }
};

#define TSB_BESSEL_ALIASES(Name, KIND)                                      \
  template <typename T> using Name##Fwd = BesselFwd<KIND, T>;              \
  template <typename T> using Name##Bwd = BesselBwd<KIND, T>;              \
  template <typename T> using Name##BwdBwd = BesselBwdBwd<KIND, T>;

TSB_BESSEL_ALIASES(BesselJ, kBJ)
TSB_BESSEL_ALIASES(BesselY, kBY)
TSB_BESSEL_ALIASES(BesselI, kBI)
TSB_BESSEL_ALIASES(BesselK, kBK)

}  // namespace tsb

namespace tsb {

// ---- integer orders 0 and 1 as unary ops: bessel_j_1, bessel_y_0, bessel_y_1,
// modified_bessel_i_0, modified_bessel_i_1, modified_bessel_k_0, modified_bessel_k_1.
// Values, first and second derivatives with the reference's conventions
// (bessel_j_1.h:93-117, bessel_y_0.h:95-116, bessel_y_1.h:94-116,
// modified_bessel_i_0.h:71-86, modified_bessel_i_1.h:55-74,
// modified_bessel_k_0.h:50-76, modified_bessel_k_1.h:51-78 and their
// _backward / _backward_backward files): Y and K are NaN for z < 0 and
// ∓inf / +inf at 0 with NaN derivatives there; J1, I1 are odd and I0 even;
// J1'(0) = I1'(0) = 1/2, J1''(0) = I1''(0) = 0, I0''(0) = 1/2.  J1 comes
// from the order-0/1 path, the others from the real-order evaluator at
// ν = 0, 1; second derivatives from Bessel's equation.
struct BesselIntVals {
  double v, d, d2;
};

template <int KIND, int ORDER>
__device__ inline BesselIntVals bessel_int_vals(double z, bool need_d2) {
  const double nan = CUDART_NAN, inf = CUDART_INF;
  if (isnan(z)) return {z, z, z};
  if (KIND == kBY || KIND == kBK) {
    if (z < 0.0) return {nan, nan, nan};
    if (z == 0.0) return {KIND == kBY ? -inf : inf, nan, nan};
  }
  if (z == 0.0) {  // J1, I0, I1
    if (KIND == kBI && ORDER == 0) return {1.0, 0.0, 0.5};
    return {0.0, 0.5, 0.0};
  }
  BV<double> b;
  if (KIND == kBJ) {
    if (isinf(z)) return {0.0, 0.0, 0.0};
    const J01 r = bessel_j01<true, true, TSB_B01_UNROLL>(z);
    b = {r.j1, r.j0 - r.j1 / z};
  } else {
    b = bessel_eval<double, KIND>((double)ORDER, z);
  }
  const double d2 = need_d2 ? (isinf(z) ? (KIND == kBI ? inf : 0.0) : bessel_d2<double, KIND>((double)ORDER, z, b)) : 0.0;
  return {b.v, b.d, d2};
}

// Region of an integer-order element (the evaluator's method for z, as in
// bessel_classify), so that the map kernel groups each warp's lanes by method:
// the real-order evaluator runs a series, Steed's fractions or Hankel's sums
// depending on z, and a warp holding all three runs all three.
template <int KIND, int ORDER>
__device__ __forceinline__ int bessel_int_classify(double z) {
  return bessel_classify<KIND>((double)ORDER, z);
}
// J1 runs the order-0/1 path, of uniform cost: one region (no staging).
template <int KIND>
constexpr int kBesselIntRegions = KIND == kBJ ? 1 : kBsRegions;

template <int KIND, int ORDER, typename T_>
struct BesselIntFwd {
  using T = T_;
  static constexpr int NIN = 1, NOUT = 1, R = kBesselIntRegions<KIND>;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) { return bessel_int_classify<KIND, ORDER>((double)in[0]); }
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    out[0] = (T)bessel_int_vals<KIND, ORDER>((double)in[0], false).v;
  }
};
template <int KIND, int ORDER, typename T_>
struct BesselIntBwd {  // in = {grad, z}
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = kBesselIntRegions<KIND>;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) { return bessel_int_classify<KIND, ORDER>((double)in[1]); }
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    out[0] = (T)((double)in[0] * bessel_int_vals<KIND, ORDER>((double)in[1], false).d);
  }
};
template <int KIND, int ORDER, typename T_>
struct BesselIntBwdBwd {  // in = {gg, grad, z}: {gg·f'(z), gg·grad·f''(z)}
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = kBesselIntRegions<KIND>;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) { return bessel_int_classify<KIND, ORDER>((double)in[2]); }
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double gg = in[0], g = in[1];
    const BesselIntVals f = bessel_int_vals<KIND, ORDER>((double)in[2], true);
    out[0] = (T)(gg * f.d);
    out[1] = (T)(gg * g * f.d2);
  }
};

#define TSB_BESSEL_INT_ALIASES(Name, KIND, ORDER)                                          \
  template <typename T> using Name##Fwd = BesselIntFwd<KIND, ORDER, T>;                 \
  template <typename T> using Name##Bwd = BesselIntBwd<KIND, ORDER, T>;                 \
  template <typename T> using Name##BwdBwd = BesselIntBwdBwd<KIND, ORDER, T>;
TSB_BESSEL_INT_ALIASES(BesselJ1, kBJ, 1)
TSB_BESSEL_INT_ALIASES(BesselY0, kBY, 0)
TSB_BESSEL_INT_ALIASES(BesselY1, kBY, 1)
TSB_BESSEL_INT_ALIASES(ModifiedBesselI0, kBI, 0)
TSB_BESSEL_INT_ALIASES(ModifiedBesselI1, kBI, 1)
TSB_BESSEL_INT_ALIASES(ModifiedBesselK0, kBK, 0)
TSB_BESSEL_INT_ALIASES(ModifiedBesselK1, kBK, 1)
#undef TSB_BESSEL_INT_ALIASES

}  // namespace tsb
