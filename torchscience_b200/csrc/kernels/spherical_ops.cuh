// Spherical Bessel functions of order 0 and 1 as unary ops:
// spherical_bessel_{j,y,i,k}_{0,1}, forward, backward and double backward.
//
// The reference evaluates closed forms (spherical_bessel_j_0.h:33-44,
// _j_1.h:33-45, _y_0.h:33-41, _y_1.h:33-42, _i_0.h:33-47, _i_1.h:33-45,
// _k_0.h:33-49, _k_1.h:33-46), with short series below |z| = 1e-12, and
// their derivatives from the recurrences (the _backward files).  Here the
// closed forms are kept where they are exact in floating point:
//   j0 = sin z / z, y0 = -cos z / z, y1 = -cos z / z² - sin z / z,
//   i0 = sinh z / z, k0 = (π/2) e^-z / z, k1 = (π/2)(1 + z) e^-z / z²,
// while j1 = sin z/z² - cos z/z and i1 = cosh z/z - sinh z/z² (and the
// derivatives that subtract 1/z terms) cancel for small |z|: below |z| = 1
// the power series of j_n, i_n (n = 0, 1) gives value and both derivatives
// (DLMF 10.53.1: j_n = z^n Σ (-z²/2)^k / (k! (2n+2k+1)!!), i_n with +z²/2).
// Second derivatives elsewhere come from the spherical Bessel equations
// z² f'' + 2z f' ± (z² ∓ n(n+1)) f = 0 (DLMF 10.47.1, 10.47.2).
// The reference's conventions: j0(0) = i0(0) = 1, j1(0) = i1(0) = 0;
// y0, y1 = -inf at 0 with NaN derivatives; k0 ~ π/(2z), k1 = +inf below
// |z| = 1e-12; negative z follows the closed forms.
#pragma once

#include <math_constants.h>

#include "dispatch.cuh"

namespace tsb {

enum SphKind : int { kSphJ = 0, kSphY = 1, kSphI = 2, kSphK = 3 };

struct SphVals {
  double v, d, d2;
};

// Series of j_n (SIGN = -1) or i_n (SIGN = +1), n = 0, 1, with d/dz and d²/dz², |z| < 1.
// f = Σ u_k z^(2k+n), u_k = (±1/2)^k / (k! (2n+2k+1)!!).  With f_k = u_k z^(2k-2)
// (k >= 1) and p = 2k + n the sums S0 = Σ f_k, S1 = Σ p f_k, S2 = Σ p(p-1) f_k
// give the value and both derivatives without dividing by z:
//   n = 0: f = u_0 + z² S0, f' = z S1, f'' = S2;
//   n = 1: f = z (u_0 + z² S0), f' = u_0 + z² S1, f'' = z S2.
// Twelve terms: at |z| < 1 the thirteenth is below 1e-20 of the first.
template <int SIGN, int ORDER>
__device__ inline SphVals sph_series(double z) {
  const double u0 = ORDER == 0 ? 1.0 : 1.0 / 3.0;
  const double h = SIGN * 0.5 * z * z;
  double f = SIGN * 0.5 * u0 / (2.0 * ORDER + 3.0);  // u_1
  double S0 = 0.0, S1 = 0.0, S2 = 0.0;
#pragma unroll
  for (int k = 1; k <= 12; ++k) {
    const double p = 2.0 * k + ORDER;
    S0 += f;
    S1 = fma(f, p, S1);
    S2 = fma(f, p * (p - 1.0), S2);
    f *= h / ((k + 1.0) * (2.0 * ORDER + 2.0 * k + 3.0));
  }
  const double z2 = z * z;
  if (ORDER == 0) return {fma(z2, S0, u0), z * S1, S2};
  return {z * fma(z2, S0, u0), fma(z2, S1, u0), z * S2};
}

template <int KIND, int ORDER>
__device__ inline SphVals sph01_vals(double z, bool need_d2) {
  const double nan = CUDART_NAN, inf = CUDART_INF, hpi = 1.5707963267948966;
  if (isnan(z)) return {z, z, z};
  const double az = fabs(z);
  if ((KIND == kSphJ || KIND == kSphI) && az < 1.0) {
    return KIND == kSphJ ? sph_series<-1, ORDER>(z) : sph_series<1, ORDER>(z);
  }
  if (KIND == kSphY && z == 0.0) return {-inf, nan, nan};
  if (KIND == kSphK && az < 1e-12) {
    if (ORDER == 0) return {hpi / z, -hpi / (z * z), hpi / (z * z * z) * 2.0};
    return {inf, -inf, inf};
  }
  const double nn = ORDER * (ORDER + 1.0);
  double v, d;
  if (KIND == kSphJ || KIND == kSphY) {
    if (isinf(z)) return {0.0, 0.0, 0.0};
    double s, c;
    sincos(z, &s, &c);
    const double r = 1.0 / z;
    if (KIND == kSphJ) {
      const double j0 = s * r, j1 = (s * r - c) * r;
      v = ORDER == 0 ? j0 : j1;
      d = ORDER == 0 ? -j1 : j0 - 2.0 * j1 * r;
    } else {
      const double y0 = -c * r, y1 = (-c * r - s) * r;
      v = ORDER == 0 ? y0 : y1;
      d = ORDER == 0 ? -y1 : y0 - 2.0 * y1 * r;
    }
    const double d2 = need_d2 ? -2.0 * d * r - (1.0 - nn * r * r) * v : 0.0;
    return {v, d, d2};
  }
  if (KIND == kSphI) {
    if (isinf(z)) return {ORDER == 0 ? inf : z, z > 0.0 ? inf : (ORDER == 0 ? -inf : inf), inf};
    // |z| >= 1: sinh, cosh without cancellation; beyond 710 the quotient overflows as the function does
    const double sh = sinh(z), ch = cosh(z), r = 1.0 / z;
    const double i0 = sh * r, i1 = (ch - sh * r) * r;
    v = ORDER == 0 ? i0 : i1;
    d = ORDER == 0 ? i1 : i0 - 2.0 * i1 * r;
    const double d2 = need_d2 ? -2.0 * d * r + (1.0 + nn * r * r) * v : 0.0;
    return {v, d, d2};
  }
  // k
  if (isinf(z)) return z > 0.0 ? SphVals{0.0, -0.0, 0.0} : SphVals{nan, nan, nan};
  const double r = 1.0 / z, e = hpi * exp(-z) * r;
  const double k0 = e, k1 = e * (1.0 + z) * r;
  v = ORDER == 0 ? k0 : k1;
  d = ORDER == 0 ? -k1 : -k0 - 2.0 * k1 * r;
  const double d2 = need_d2 ? -2.0 * d * r + (1.0 + nn * r * r) * v : 0.0;
  return {v, d, d2};
}

template <int KIND, int ORDER, typename T_>
struct Sph01Fwd {
  using T = T_;
  static constexpr int NIN = 1, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    out[0] = (T)sph01_vals<KIND, ORDER>((double)in[0], false).v;
  }
};
template <int KIND, int ORDER, typename T_>
struct Sph01Bwd {  // in = {grad, z}
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    out[0] = (T)((double)in[0] * sph01_vals<KIND, ORDER>((double)in[1], false).d);
  }
};
template <int KIND, int ORDER, typename T_>
struct Sph01BwdBwd {  // in = {gg, grad, z}: {gg·f', gg·grad·f''}
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = 1;
  static constexpr bool REDUCE = true;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double gg = in[0], g = in[1];
    const SphVals f = sph01_vals<KIND, ORDER>((double)in[2], true);
    out[0] = (T)(gg * f.d);
    out[1] = (T)(gg * g * f.d2);
  }
};

#define TSB_SPH01_ALIASES(Name, KIND, ORDER)                                   \
  template <typename T> using Name##Fwd = Sph01Fwd<KIND, ORDER, T>;          \
  template <typename T> using Name##Bwd = Sph01Bwd<KIND, ORDER, T>;          \
  template <typename T> using Name##BwdBwd = Sph01BwdBwd<KIND, ORDER, T>;
TSB_SPH01_ALIASES(SphJ0, kSphJ, 0)
TSB_SPH01_ALIASES(SphJ1, kSphJ, 1)
TSB_SPH01_ALIASES(SphY0, kSphY, 0)
TSB_SPH01_ALIASES(SphY1, kSphY, 1)
TSB_SPH01_ALIASES(SphI0, kSphI, 0)
TSB_SPH01_ALIASES(SphI1, kSphI, 1)
TSB_SPH01_ALIASES(SphK0, kSphK, 0)
TSB_SPH01_ALIASES(SphK1, kSphK, 1)
#undef TSB_SPH01_ALIASES

}  // namespace tsb

// ---- spherical Bessel functions of real order n: spherical_bessel_{j,y,i,k}(n, z)
// f_n(z) = sqrt(π/(2|z|)) C_{n+1/2}(|z|) with C = J, Y, I, K (DLMF 10.47.3, 10.47.7,
// 10.47.8 with the reference's normalisation of k), evaluated by the real-order
// Bessel evaluators, with the reference's conventions (spherical_bessel_j.h,
// _y.h, _i.h, _k.h; the `spherical_bessel_*(T n, T z)` functions):
//   - n within 1e-12 of an integer counts as that integer; |z| < 1e-12 counts
//     as 0: j, i = 1 at n = 0, 0 for n > 0, inf for n < 0; y = -inf; k = +inf;
//     ∂/∂z there: j, i 0 (1/3 at n = 1, NaN for n < 0); y, k -inf;
//   - z < 0: k is NaN; j, i take the factor (-1)^n for integer n and cos(πn)
//     otherwise, y the factor (-1)^(n+1) or cos(π(n+1));
//   - ∂/∂n by central differences of this function (step ε^(1/3) max(1, |n|),
//     ε^(1/4) for the second derivative), as the reference differentiates in n
//     numerically; ∂/∂z from the evaluator (below |z| = 1 from the order
//     recurrence, since C' - C/(2z) cancels there), ∂²/∂z² from the spherical
//     Bessel equation.

#include "bessel_ops.cuh"

namespace tsb {

constexpr double kSphEps = 1e-12;

template <int KIND>
__device__ inline double sph_phase(double n) {  // factor for z < 0 (j, y, i)
  const double nr = rint(n);
  const double m = KIND == kSphY ? 1.0 : 0.0;
  if (fabs(n - nr) < kSphEps) return fmod(fabs(nr + m), 2.0) == 1.0 ? -1.0 : 1.0;
  double s, c;
  sincospi(n + m, &s, &c);
  return c;
}

// f_n(z) and ∂f/∂z (and, when D2, ∂²f/∂z²) with the conventions above.
template <int KIND, bool D2>
__device__ inline SphVals sph_eval(double n, double z) {
  const double nan = CUDART_NAN, inf = CUDART_INF;
  if (isnan(n) || isnan(z)) return {nan, nan, nan};
  if (fabs(z) < kSphEps) {
    double v;
    if (KIND == kSphY) v = -inf;
    else if (KIND == kSphK) v = inf;
    else v = fabs(n) < kSphEps ? 1.0 : (n > 0.0 ? 0.0 : inf);
    double d = -inf;  // y, k: the reference's value at the pole
    if (KIND == kSphJ || KIND == kSphI) d = fabs(n) < kSphEps ? 0.0 : (fabs(n - 1.0) < kSphEps ? 1.0 / 3.0 : (n > 0.0 ? 0.0 : nan));
    return {v, d, nan};
  }
  if (KIND == kSphK && z < 0.0) return {nan, nan, nan};
  const double nr = rint(n);
  const double nn = (n >= 0.0 && fabs(n - nr) < kSphEps) ? nr : n;  // the order used
  const double az = fabs(z), nu = nn + 0.5;
  BV<double> b;
  if (KIND == kSphJ) b = bessel_eval<double, kBJ>(nu, az);
  else if (KIND == kSphY) b = bessel_eval<double, kBY>(nu, az);
  else if (KIND == kSphI) b = bessel_eval<double, kBI>(nu, az);
  else b = bessel_eval<double, kBK>(nu, az);
  if (isinf(az)) return {b.v == b.v ? (KIND == kSphI ? b.v : 0.0) : nan, 0.0, 0.0};
  const double pre = sqrt(1.5707963267948966 / az);
  double v = pre * b.v, d;
  if (az < 1.0) {
    // C' - C/(2z) cancels as z -> 0: the order recurrence instead,
    // d/dz [pre C_ν] = pre ((n/z) C_ν - C_{ν+1}) (J, Y, K), pre ((n/z) I_ν + I_{ν+1}) (I)
    double c1;
    if (KIND == kSphJ) c1 = bessel_eval<double, kBJ>(nu + 1.0, az).v;
    else if (KIND == kSphY) c1 = bessel_eval<double, kBY>(nu + 1.0, az).v;
    else if (KIND == kSphI) c1 = bessel_eval<double, kBI>(nu + 1.0, az).v;
    else c1 = bessel_eval<double, kBK>(nu + 1.0, az).v;
    d = pre * fma(nn / az, b.v, KIND == kSphI ? c1 : -c1);
  } else {
    d = pre * (b.d - 0.5 * b.v / az);
  }
  double d2 = 0.0;
  if (D2) {
    const double r = 1.0 / az, q = nn * (nn + 1.0) * r * r;
    d2 = (KIND == kSphJ || KIND == kSphY) ? -2.0 * d * r - (1.0 - q) * v : -2.0 * d * r + (1.0 + q) * v;
  }
  if (z < 0.0) {  // f(z) = φ g(|z|): f' = -φ g', f'' = φ g''
    const double ph = sph_phase<KIND>(n);
    v *= ph;
    d *= -ph;
    d2 *= ph;
  }
  return {v, d, d2};
}

struct SphNuDerivs {
  double dn, dnz, dnn;  // ∂f/∂n, ∂²f/∂n∂z, ∂²f/∂n²
};
template <int KIND, bool SECOND>
__device__ inline SphNuDerivs sph_nu_derivs(double n, double z, double f0) {
  SphNuDerivs o{0.0, 0.0, 0.0};
  const double h = 6.0554544523933395e-06 * fmax(1.0, fabs(n));
  const SphVals p = sph_eval<KIND, false>(n + h, z), m = sph_eval<KIND, false>(n - h, z);
  o.dn = (p.v - m.v) / (2.0 * h);
  o.dnz = (p.d - m.d) / (2.0 * h);
  if (SECOND) {
    const double h2 = 1.2207031250e-04 * fmax(1.0, fabs(n));
    const double vp = sph_eval<KIND, false>(n + h2, z).v, vm = sph_eval<KIND, false>(n - h2, z).v;
    o.dnn = (vp - 2.0 * f0 + vm) / (h2 * h2);
  }
  return o;
}

// Region of (n, z): the real-order evaluator's method at order n + 1/2 and
// |z| (bessel_classify), so that the map kernel groups each warp's lanes by
// method.
template <int KIND>
__device__ __forceinline__ int sph_classify(double n, double z) {
  if (isnan(n) || isnan(z) || fabs(z) < kSphEps) return kBsSpecial;
  constexpr int KB = KIND == kSphJ ? kBJ : KIND == kSphY ? kBY : KIND == kSphI ? kBI : kBK;
  return bessel_classify<KB>(n + 0.5, fabs(z));
}

template <int KIND, typename T_>
struct SphFwd {  // in = {n, z}
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = kBsRegions;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) { return sph_classify<KIND>((double)in[0], (double)in[1]); }
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    out[0] = (T)sph_eval<KIND, false>((double)in[0], (double)in[1]).v;
  }
};
template <int KIND, typename T_>
struct SphBwd {  // in = {grad, n, z}, out = {grad_n, grad_z}
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = kBsRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) { return sph_classify<KIND>((double)in[1], (double)in[2]); }
  __device__ static void eval(int, const T* in, T* out, uint32_t mask) {
    const double g = in[0], n = in[1], z = in[2];
    const SphVals f = sph_eval<KIND, false>(n, z);
    out[0] = (mask & 1u) ? (T)(g * sph_nu_derivs<KIND, false>(n, z, f.v).dn) : T(0);
    out[1] = (T)(g * f.d);
  }
};
template <int KIND, typename T_>
struct SphBwdBwd {  // in = {gg_n, gg_z, grad, n, z}, out = {grad_grad_output, grad_n, grad_z}
  using T = T_;
  static constexpr int NIN = 5, NOUT = 3, R = kBsRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) { return sph_classify<KIND>((double)in[3], (double)in[4]); }
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double ggn = in[0], ggz = in[1], g = in[2], n = in[3], z = in[4];
    const SphVals f = sph_eval<KIND, true>(n, z);
    const SphNuDerivs dn = sph_nu_derivs<KIND, true>(n, z, f.v);
    out[0] = (T)(ggn * dn.dn + ggz * f.d);
    out[1] = (T)(g * (ggn * dn.dnn + ggz * dn.dnz));
    out[2] = (T)(g * (ggn * dn.dnz + ggz * f.d2));
  }
};

#define TSB_SPH_ALIASES(Name, KIND)                                   \
  template <typename T> using Name##Fwd = SphFwd<KIND, T>;           \
  template <typename T> using Name##Bwd = SphBwd<KIND, T>;           \
  template <typename T> using Name##BwdBwd = SphBwdBwd<KIND, T>;
TSB_SPH_ALIASES(SphJ, kSphJ)
TSB_SPH_ALIASES(SphY, kSphY)
TSB_SPH_ALIASES(SphI, kSphI)
TSB_SPH_ALIASES(SphK, kSphK)
#undef TSB_SPH_ALIASES

}  // namespace tsb
