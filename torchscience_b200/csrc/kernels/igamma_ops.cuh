// Regularized incomplete gamma P(a,x) and Q(a,x) = 1 - P: functors of the
// forward, backward (grad_a, grad_x) and double-backward entry points.  Output conventions
// follow regularized_gamma_p_backward.h:27-33 and
// regularized_gamma_p_backward_backward.h:12-41 (Q negates every derivative,
// regularized_gamma_q_backward_backward.h:16-21).
#pragma once

#include "dispatch.cuh"
#include "igamma_math.cuh"
#include "stream2d.cuh"
#include "sweep.cuh"

// Resident CTAs the forward's register allocation must allow (64 registers).
#ifndef TSB_IGF_MINB
#define TSB_IGF_MINB 4
#endif


namespace tsb {

// ∂P/∂x alone (backward with grad_a not requested): no series needed.
__device__ __forceinline__ double igamma_px_only(double a, double x, const IgPre& P) {
  if (isnan(a) || isnan(x) || x < 0.0 || a <= 0.0) return CUDART_NAN;
  if (x == 0.0 || isinf(x) || isinf(a)) return 0.0;
  // the same expressions as the full backward (igamma_eval_d), branch by branch
  const double lnD = igamma_log_prefix_d(a, x, P);
  if (x < a + 1.0) return igamma_px_from(exp(lnD), lnD, a, P);
  const double lnE = lnD + P.la();
  return lnE > -700.0 ? exp(lnE) * P.rx() : exp(lnE - P.lx());
}

// Every functor here keeps per-row / per-column tables of its a and x inputs
// (a quantities: lnΓ or the Stirling constant, ln a, 1/a, ψ(a), ψ'(a) and the
// classifier's float values; x: ln x), which the 2-D kernel fills once per
// tile row or column when the input is broadcast along the other dimension.
template <int ORDER, int IA, int IX, typename T>
struct IgammaAuxIO {
  static constexpr int AUX_IN0 = IA, AUX_IN1 = IX;
  static constexpr int NAUX0 = kIgAuxA, NAUX1 = kIgAuxX;
  static constexpr bool SWEEP = true;  // (R, 1) x (1, C) grids run the row-sorted sweep
  __device__ static void make_aux0(T v, double* o) { igamma_aux_a<ORDER>((double)v, o); }
  __device__ static void make_aux1(T v, double* o) { igamma_aux_x((double)v, o); }
  __device__ static IgPre pre(const T* in, const double* A, const double* X) {
    return IgPre{A, X, (double)in[IA], (double)in[IX]};
  }
  __device__ static int classify(const T* in, const double* A = nullptr, const double* X = nullptr) {
    return igamma_classify((double)in[IA], (double)in[IX], pre(in, A, X), sizeof(T) == 4 && ORDER == 0);
  }
};

// Each functor evaluates through eval_impl<UNIFORM>: the map kernel calls the
// four-argument eval (independent points: the uniform expansion takes its
// window), the kernels with per-row / per-column tables the six-argument one.
template <typename T_, bool UPPER>
struct IgammaFwd : IgammaAuxIO<0, 0, 1, T_> {
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = kIgRegions;
  static constexpr int MIN_BLOCKS = TSB_IGF_MINB;
  static constexpr bool REDUCE = false;
  template <bool UNIFORM>
  __device__ static void eval_impl(int r, const T* in, T* out, const double* A, const double* X) {
    const IgammaOut o = igamma_eval<0, UPPER, UNIFORM>(r, in[0], in[1], IgammaFwd::pre(in, A, X));
    out[0] = (T)(UPPER ? o.q : o.p);
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) { eval_impl<true>(r, in, out, nullptr, nullptr); }
  __device__ static void eval(int r, const T* in, T* out, uint32_t, const double* A, const double* X) {
    eval_impl<false>(r, in, out, A, X);
  }
};

template <typename T_, bool UPPER>
struct IgammaBwd : IgammaAuxIO<1, 1, 2, T_> {
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = kIgRegions;
  // 64 registers, 4 resident CTAs: measured 15% faster than the unconstrained
  // allocation (118 registers, 2 CTAs) on the 4096 x 4096 grid.
  static constexpr int MIN_BLOCKS = 4;
  static constexpr bool REDUCE = true;
  template <bool UNIFORM>
  __device__ static void eval_impl(int r, const T* in, T* out, uint32_t mask, const double* A, const double* X) {
    const double sgn = UPPER ? -1.0 : 1.0;
    const double g = in[0];
    const IgPre P = IgammaBwd::pre(in, A, X);
    if (!(mask & 1u)) {
      out[0] = T(0);
      out[1] = (T)(sgn * g * igamma_px_only((double)in[1], (double)in[2], P));
      return;
    }
    const IgammaOut o = igamma_eval<1, false, UNIFORM>(r, in[1], in[2], P);
    out[0] = (T)(sgn * g * o.pa);
    out[1] = (T)(sgn * g * o.px);
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t mask) {
    eval_impl<true>(r, in, out, mask, nullptr, nullptr);
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t mask, const double* A, const double* X) {
    eval_impl<false>(r, in, out, mask, A, X);
  }
  // Two-pass sweep of float data: pass 1 the FP32 elements, pass 2 the rest.
  static constexpr bool SPLIT = sizeof(T) == 4;
  // Saturated elements (every derivative 0) take the first pass.
  __device__ static bool fp64_pass(int r, const T* in, uint32_t mask, const double* A, const double* X) {
    return !(mask & 1u) || (r != kIgSat0 && r != kIgSat1 &&
                            igamma_needs_fp64_1(r, (float)in[2], IgammaBwd::pre(in, A, X), false));
  }
  template <int PASS>
  __device__ static void eval_pass(int r, const T* in, T* out, uint32_t mask, const double* A, const double* X) {
    const double sgn = UPPER ? -1.0 : 1.0;
    const double g = in[0];
    const IgPre P = IgammaBwd::pre(in, A, X);
    if constexpr (PASS == 1) {
      const IgammaOut o = (r == kIgSat0 || r == kIgSat1) ? igamma_saturated(r == kIgSat1)
                                                         : igamma_eval_mf1<false>(r, (float)in[1], (float)in[2], P);
      out[0] = (T)(sgn * g * o.pa);
      out[1] = (T)(sgn * g * o.px);
    } else {
      if (!(mask & 1u)) {
        out[0] = T(0);
        out[1] = (T)(sgn * g * igamma_px_only((double)in[1], (double)in[2], P));
        return;
      }
      const IgammaOut o = igamma_eval<1>(r, (double)in[1], (double)in[2], P);
      out[0] = (T)(sgn * g * o.pa);
      out[1] = (T)(sgn * g * o.px);
    }
  }
};

template <typename T_, bool UPPER>
struct IgammaBwdBwd : IgammaAuxIO<2, 3, 4, T_> {
  using T = T_;
  static constexpr int NIN = 5, NOUT = 3, R = kIgRegions;
  static constexpr bool REDUCE = true;
  __device__ static void eval(int r, const T* in, T* out, uint32_t, const double* A = nullptr,
                              const double* X = nullptr) {
    const double sgn = UPPER ? -1.0 : 1.0;
    const double gga = in[0], ggx = in[1], g = in[2];
    const IgammaOut o = igamma_eval<2>(r, in[3], in[4], IgammaBwdBwd::pre(in, A, X));
    // sums of two products as explicit fmas, so that every kernel that
    // instantiates this functor rounds them the same way (the compiler may
    // otherwise contract either product)
    out[0] = (T)(sgn * fma(gga, o.pa, __dmul_rn(ggx, o.px)));
    out[1] = (T)(sgn * g * fma(gga, o.paa, __dmul_rn(ggx, o.pax)));
    out[2] = (T)(sgn * g * fma(gga, o.pax, __dmul_rn(ggx, o.pxx)));
  }
};

// Forward with the first derivatives, for autograd: in = {a, x}, out =
// {P (or Q), ∂/∂a, ∂/∂x} at full shape, in one evaluation.  A training step
// that differentiates P otherwise evaluates the series or fraction twice, once
// for the value and again in the backward; here the backward only multiplies
// the kept derivatives by its incoming gradient (GradProduct).  ∂/∂a is
// skipped when its output is not requested (then ∂/∂x alone, as in the
// backward above).
#ifndef TSB_IGFG_TR
#define TSB_IGFG_TR 64
#endif
template <typename T_, bool UPPER>
struct IgammaFwdGrad : IgammaAuxIO<1, 0, 1, T_> {
  using T = T_;
  static constexpr int NIN = 2, NOUT = 3, R = kIgRegions;
  static constexpr int MIN_BLOCKS = 4;
  static constexpr int TILE_ROWS = TSB_IGFG_TR;
  static constexpr bool REDUCE = false;
  // Float data is evaluated in FP64 here as well, and stored as float.  On
  // the configuration-2 workload the mixed alternatives measured slower: the
  // two-pass split of the sweep (an FP32 pass for the light elements, an
  // FP64 pass for the rest) 0.77 ms against 0.62 ms for one FP64 pass, since
  // the FP32 pass saves little on elements whose FP64 cost is a few series
  // terms and one exponential; and the mixed evaluators on the 2^20
  // transition points 118 us against 105 us.  The forward without
  // derivatives keeps the mixed evaluators (1.2x FP64).
  template <bool UNIFORM>
  __device__ static void eval_impl(int r, const T* in, T* out, uint32_t mask, const double* A, const double* X) {
    const double sgn = UPPER ? -1.0 : 1.0;
    const IgPre P = IgammaFwdGrad::pre(in, A, X);
    const double a = (double)in[0], x = (double)in[1];
    if (!(mask & 2u)) {
      const IgammaOut o = igamma_eval<0, UPPER, UNIFORM>(r, a, x, P);
      out[0] = (T)(UPPER ? o.q : o.p);
      out[1] = T(0);
      out[2] = (T)(sgn * igamma_px_only(a, x, P));
      return;
    }
    const IgammaOut o = igamma_eval<1, UPPER, UNIFORM>(r, a, x, P);
    out[0] = (T)(UPPER ? o.q : o.p);
    out[1] = (T)(sgn * o.pa);
    out[2] = (T)(sgn * o.px);
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t mask) {
    eval_impl<true>(r, in, out, mask, nullptr, nullptr);
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t mask, const double* A, const double* X) {
    eval_impl<false>(r, in, out, mask, A, X);
  }
};

// Backward from kept derivatives: in = {grad, d_a, d_b}, out = {grad·d_a,
// grad·d_b}, each reduced to its input's shape by the 2-D kernel.  The
// products are formed in double for every storage type (GradProductD), so
// a reduced gradient of float data is rounded once, after the sum, as the
// reference's backward op rounds each product once
// (regularized_gamma_p_backward.h:27-33).
template <typename T_>
struct GradProduct {
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = 1;
  static constexpr bool REDUCE = true;
  static constexpr bool STREAM2D = true;  // HBM-bound: the streaming 2-D reduction when the layout allows
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    out[0] = in[0] * in[1];
    out[1] = in[0] * in[2];
  }
};

template <typename T> using GradProductD = GradProduct<double>;
template <typename T> using GammaPFwd = IgammaFwd<T, false>;
template <typename T> using GammaPBwd = IgammaBwd<T, false>;
template <typename T> using GammaPBwdBwd = IgammaBwdBwd<T, false>;
template <typename T> using GammaQFwd = IgammaFwd<T, true>;
template <typename T> using GammaQBwd = IgammaBwd<T, true>;
template <typename T> using GammaQBwdBwd = IgammaBwdBwd<T, true>;
template <typename T> using GammaPFwdGrad = IgammaFwdGrad<T, false>;
template <typename T> using GammaQFwdGrad = IgammaFwdGrad<T, true>;

}  // namespace tsb
