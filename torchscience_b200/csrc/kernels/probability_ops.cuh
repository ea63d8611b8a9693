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
#pragma once

#include "dispatch.cuh"
#include "igamma_math.cuh"

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

}  // namespace tsb
