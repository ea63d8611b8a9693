// Gauss hypergeometric 2F1(a, b; c; z): functors of the forward, backward
// (grad_a, grad_b, grad_c, grad_z) and double-backward entry points.  Output
// conventions follow hypergeometric_2_f_1_backward.h:60-118 and
// hypergeometric_2_f_1_backward_backward.h:12-125 (gg_out, then the new
// grads in argument order).  Every precision evaluates in FP64 (the
// connection formulas cancel by up to ~1e3 on the benchmark domain, beyond
// what an FP32 bulk can absorb at 1e-6) and stores in the data type.  The
// backward declines the elements whose connection formula cancels (the
// evaluator search and its long direct series with derivatives) to the map
// kernel's rescue list, which evaluates them in full warps after the tile:
// 1.7x on the benchmark's fwd + grads.  The forward keeps them in place: its
// declined elements would evaluate the connection formula twice, which
// measured 35% slower.
#pragma once

#include "dispatch.cuh"
#include "hyp2f1_math.cuh"

// Resident CTAs the forward and backward register allocation must allow: 4
// (64 registers, with spills) measured 25% faster forward and 15% faster
// backward than the unconstrained allocation (122 / 200 registers).
#ifndef TSB_H2_MINB
#define TSB_H2_MINB 4
#endif

namespace tsb {

// The reference's special-case tolerance for the data type (hyp2f1_epsilon).
template <typename T>
__device__ constexpr double h2f1_eps_for() {
  return sizeof(T) == 8 ? 1e-15 : 1e-7;
}

template <typename T_>
struct Hyp2f1Fwd {
  using T = T_;
  static constexpr int MIN_BLOCKS = TSB_H2_MINB;
  static constexpr int NIN = 4, NOUT = 1, R = kH2Regions;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) {
    return h2f1_classify((double)in[0], (double)in[1], (double)in[2], (double)in[3], h2f1_eps_for<T>());
  }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) {
    const double a = in[0], b = in[1], c = in[2], z = in[3];
    double v;
    if (r == kH2Special) {
      h2f1_special(a, b, c, z, v, h2f1_eps_for<T>());
    } else {
      v = h2f1_eval(r, a, b, c, z);
    }
    out[0] = (T)v;
  }
};

template <typename T_>
struct Hyp2f1Bwd {
  using T = T_;
  static constexpr int MIN_BLOCKS = TSB_H2_MINB;
  static constexpr int NIN = 5, NOUT = 4, R = kH2Regions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) {
    return h2f1_classify((double)in[1], (double)in[2], (double)in[3], (double)in[4], h2f1_eps_for<T>());
  }
  __device__ static void eval(int, const T* in, T* out, uint32_t mask) {
    const double g = in[0], a = in[1], b = in[2], c = in[3], z = in[4];
    if (!(mask & 7u)) {  // grad_z alone
      out[0] = out[1] = out[2] = T(0);
      out[3] = (T)(g * h2f1_dz(a, b, c, z, h2f1_eps_for<T>()));
      return;
    }
    store(g, h2f1_grad(a, b, c, z, h2f1_eps_for<T>()), out);
  }
  __device__ static void store(double g, const H2f1Grad& d, T* out) {
    out[0] = (T)(g * d.da);
    out[1] = (T)(g * d.db);
    out[2] = (T)(g * d.dc);
    out[3] = (T)(g * d.dz);
  }
  // Elements whose connection formula cancels go through the rescue list.
  static constexpr bool RESCUE = true;
  __device__ static bool eval_first(int r, const T* in, T* out, uint32_t mask) {
    if (!(mask & 7u)) {
      eval(r, in, out, mask);
      return true;
    }
    H2f1Grad d;
    if (!h2f1_grad_first((double)in[1], (double)in[2], (double)in[3], (double)in[4], h2f1_eps_for<T>(), d))
      return false;
    store((double)in[0], d, out);
    return true;
  }
  __device__ static void eval_rescue(int, const T* in, T* out, uint32_t) {
    store((double)in[0], h2f1_grad_fallback((double)in[1], (double)in[2], (double)in[3], (double)in[4]), out);
  }
};

template <typename T_>
struct Hyp2f1BwdBwd {
  using T = T_;
  static constexpr int NIN = 9, NOUT = 5, R = kH2Regions;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) {
    return h2f1_classify((double)in[5], (double)in[6], (double)in[7], (double)in[8], h2f1_eps_for<T>());
  }
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const double gg[4] = {in[0], in[1], in[2], in[3]};
    const double g = in[4];
    const H2f1Hess H = h2f1_hessian((double)in[5], (double)in[6], (double)in[7], (double)in[8], h2f1_eps_for<T>());
    // packed [aa, ab, ac, az, bb, bc, bz, cc, cz, zz]
    const double M[4][4] = {{H.h[0], H.h[1], H.h[2], H.h[3]},
                            {H.h[1], H.h[4], H.h[5], H.h[6]},
                            {H.h[2], H.h[5], H.h[7], H.h[8]},
                            {H.h[3], H.h[6], H.h[8], H.h[9]}};
    out[0] = (T)(gg[0] * H.g.da + gg[1] * H.g.db + gg[2] * H.g.dc + gg[3] * H.g.dz);
#pragma unroll
    for (int i = 0; i < 4; ++i)
      out[1 + i] = (T)(g * (gg[0] * M[i][0] + gg[1] * M[i][1] + gg[2] * M[i][2] + gg[3] * M[i][3]));
  }
};

}  // namespace tsb
