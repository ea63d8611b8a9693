// Probability callers of the regularized incomplete gamma: the gamma, χ² and
// Poisson cumulative distributions with their backward passes.  They follow
// the reference's kernels:
//   gamma_cumulative_distribution.h:9-13 (F = P(shape, x/scale), 0 for x <= 0),
//   gamma_cumulative_distribution_backward.h:16-43,
//   chi2_cumulative_distribution.h:9-13 (F = P(df/2, x/2)),
//   chi2_cumulative_distribution_backward.h:11-37,
//   poisson_cumulative_distribution.h:10-18 (F = Q(floor(k)+1, rate), 0 for k < 0),
//   poisson_cumulative_distribution_backward.h:13-29 (d/dk = 0).
// The a-derivatives are analytic here (the reference differentiates P
// numerically, regularized_gamma_p_backward.h:19-25).
//
// Also the χ² survival function Q(df/2, x/2) (chi2_survival.h:9-13,
// chi2_survival_backward.h:11-17; Q directly, not 1 - P) and the gamma and χ²
// densities (gamma_probability_density.h:9-16, *_backward.h:17-40;
// chi2_probability_density.h:10-21, *_backward.h:11-40).  The densities
// are ∂P/∂x of the incomplete gamma at t = x/scale (or x/2), with the
// Temme form of the prefactor for large shapes, instead of the reference's
// exp((shape-1) ln x - x/scale - shape ln scale - lnΓ(shape)), which loses
// relative accuracy in proportion to the size of those terms.  The
// df-derivative of the χ² density is analytic (the reference uses a central
// difference with step sqrt(ε)·max(1, |df|)).
#pragma once

#include "dispatch.cuh"
#include "igamma_ops.cuh"

namespace tsb {

// ---- gamma(x; shape, scale) -------------------------------------------------
template <typename T_>
struct GammaCdfFwd {
  using T = T_;
  static constexpr int NIN = 3, NOUT = 1, R = kIgRegions;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) {
    const double x = in[0];
    return x <= 0.0 ? kIgSpecial : igamma_classify((double)in[1], x / (double)in[2]);
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) {
    const double x = in[0];
    if (x <= 0.0) {
      out[0] = T(0);
      return;
    }
    out[0] = (T)igamma_eval<0>(r, (double)in[1], x / (double)in[2]).p;
  }
};

template <typename T_>
struct GammaCdfBwd {
  using T = T_;
  static constexpr int NIN = 4, NOUT = 3, R = kIgRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) {
    const double x = in[1];
    return x <= 0.0 ? kIgSpecial : igamma_classify((double)in[2], x / (double)in[3]);
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) {
    const double g = in[0], x = in[1], shape = in[2], scale = in[3];
    if (x <= 0.0) {
      out[0] = out[1] = out[2] = T(0);
      return;
    }
    const IgammaOut o = igamma_eval<1>(r, shape, x / scale);
    out[0] = (T)(g * o.px / scale);                  // the density
    out[1] = (T)(g * o.pa);
    out[2] = (T)(g * o.px * (-x / (scale * scale)));
  }
};

// ---- chi2(x; df) ------------------------------------------------------------
template <typename T_>
struct Chi2CdfFwd {
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = kIgRegions;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) {
    const double x = in[0];
    return x <= 0.0 ? kIgSpecial : igamma_classify(0.5 * (double)in[1], 0.5 * x);
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) {
    const double x = in[0];
    if (x <= 0.0) {
      out[0] = T(0);
      return;
    }
    out[0] = (T)igamma_eval<0>(r, 0.5 * (double)in[1], 0.5 * x).p;
  }
};

template <typename T_>
struct Chi2CdfBwd {
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = kIgRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) {
    const double x = in[1];
    return x <= 0.0 ? kIgSpecial : igamma_classify(0.5 * (double)in[2], 0.5 * x);
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) {
    const double g = in[0], x = in[1];
    if (x <= 0.0) {
      out[0] = out[1] = T(0);
      return;
    }
    const IgammaOut o = igamma_eval<1>(r, 0.5 * (double)in[2], 0.5 * x);
    out[0] = (T)(0.5 * g * o.px);
    out[1] = (T)(0.5 * g * o.pa);
  }
};

// ---- poisson(k; rate) -------------------------------------------------------
template <typename T_>
struct PoissonCdfFwd {
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = kIgRegions;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) {
    const double k = floor((double)in[0]);
    return k < 0.0 ? kIgSpecial : igamma_classify(k + 1.0, (double)in[1]);
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) {
    const double k = floor((double)in[0]);
    if (k < 0.0) {
      out[0] = T(0);
      return;
    }
    out[0] = (T)igamma_eval<0, true>(r, k + 1.0, (double)in[1]).q;
  }
};

template <typename T_>
struct PoissonCdfBwd {
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = kIgRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) {
    const double k = floor((double)in[1]);
    return k < 0.0 ? kIgSpecial : igamma_classify(k + 1.0, (double)in[2]);
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) {
    const double g = in[0], k = floor((double)in[1]);
    out[0] = T(0);
    if (k < 0.0) {
      out[1] = T(0);
      return;
    }
    // dQ/dx = -dP/dx
    out[1] = (T)(-g * igamma_eval<1>(r, k + 1.0, (double)in[2]).px);
  }
};

// ---- chi2 survival: Q(df/2, x/2), 1 for x <= 0 ----------------------------
template <typename T_>
struct Chi2SurvivalFwd {
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = kIgRegions;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) { return Chi2CdfFwd<T>::classify(in); }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) {
    const double x = in[0];
    if (x <= 0.0) {
      out[0] = T(1);
      return;
    }
    out[0] = (T)igamma_eval<0, true>(r, 0.5 * (double)in[1], 0.5 * x).q;
  }
};

template <typename T_>
struct Chi2SurvivalBwd {
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = kIgRegions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) { return Chi2CdfBwd<T>::classify(in); }
  __device__ static void eval(int r, const T* in, T* out, uint32_t mask) {
    Chi2CdfBwd<T>::eval(r, in, out, mask);
    out[0] = -out[0];
    out[1] = -out[1];
  }
};

// ---- densities ---------------------------------------------------------------
// t^(a-1) e^(-t) / Γ(a) for t > 0 (∂P/∂t), from the same expressions as the
// incomplete-gamma backward.
__device__ __forceinline__ double gamma_density_std(double a, double t) {
  return igamma_px_only(a, t, IgPre{nullptr, nullptr, a, t});
}

template <typename T_>
struct GammaPdfFwd {  // in = {x, shape, scale}
  using T = T_;
  static constexpr int NIN = 3, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double x = in[0], a = in[1], s = in[2];
    out[0] = x <= 0.0 ? T(0) : (T)(gamma_density_std(a, x / s) / s);
  }
};

template <typename T_>
struct GammaPdfBwd {  // in = {grad, x, shape, scale}, out = {grad_x, grad_shape, grad_scale}
  using T = T_;
  static constexpr int NIN = 4, NOUT = 3, R = 1;
  static constexpr bool REDUCE = true;
  __device__ static void eval(int, const T* in, T* out, uint32_t mask) {
    const double g = in[0], x = in[1], a = in[2], s = in[3];
    if (x <= 0.0) {
      out[0] = out[1] = out[2] = T(0);
      return;
    }
    const double t = x / s, f = gamma_density_std(a, t) / s;
    out[0] = (T)(g * f * ((a - 1.0) - t) / x);                    // f·((a-1)/x - 1/scale)
    out[1] = (mask & 2u) ? (T)(g * f * (log(t) - digamma_d(a))) : T(0);  // f·(ln(x/scale) - ψ(a))
    out[2] = (T)(g * f * (t - a) / s);                            // f·(x/scale² - a/scale)
  }
};

template <typename T_>
struct Chi2PdfFwd {  // in = {x, df}
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double x = in[0], df = in[1];
    double f;
    if (x < 0.0) f = 0.0;
    else if (x == 0.0) f = df < 2.0 ? CUDART_INF : (df == 2.0 ? 0.5 : 0.0);
    else f = 0.5 * gamma_density_std(0.5 * df, 0.5 * x);
    out[0] = (T)f;
  }
};

template <typename T_>
struct Chi2PdfBwd {  // in = {grad, x, df}, out = {grad_x, grad_df}
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = 1;
  static constexpr bool REDUCE = true;
  __device__ static void eval(int, const T* in, T* out, uint32_t mask) {
    const double g = in[0], x = in[1], k = 0.5 * (double)in[2];
    if (x <= 0.0) {
      out[0] = out[1] = T(0);
      return;
    }
    const double t = 0.5 * x, f = 0.5 * gamma_density_std(k, t);
    out[0] = (T)(g * f * ((k - 1.0) - t) / x);                              // f·((k/2-1)/x - 1/2)
    out[1] = (mask & 2u) ? (T)(0.5 * g * f * (log(t) - digamma_d(k))) : T(0);  // f·(ln(x/2) - ψ(k/2))/2
  }
};

}  // namespace tsb
