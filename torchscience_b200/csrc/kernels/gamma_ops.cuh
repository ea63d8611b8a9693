// lnΓ, Γ, ψ, ψ' — functors of the forward, backward and double-backward
// entry points.
// Reference scalar kernels: log_gamma.h, gamma.h, digamma.h, trigamma.h and
// their *_backward / *_backward_backward headers (same formulas:
// d lnΓ = ψ, dΓ = Γψ, d²Γ = Γ(ψ² + ψ'), dψ = ψ', dψ' = ψ'').
//
// FP64 kernels (double data) evaluate everything in double.  Mixed kernels
// (float/half/bf16 data) evaluate in FP32 and send the rare arguments the
// FP32 path would not hold to 1e-6 (x <= 0: reflection and the negative
// zeros) through the FP64 evaluator of the same formula.  The rescue is rare
// enough that a divergent branch costs less than staging the tile through
// shared memory for compaction.
#pragma once

#include <type_traits>

#include "dispatch.cuh"
#include "gamma_math.cuh"

namespace tsb {

// Per-function traits: f0 = value; s1(s, z) = s·f'(z); s2(s, z) = s·f''(z)
// (the scale s is applied where it keeps FP32 intermediates in range);
// rescue(z): FP32 argument that takes the FP64 path in the mixed kernels.
struct LogGammaFn {
  template <class T> __device__ static T f0(T z) { return lgamma_t(z); }
  template <class T> __device__ static T s1(T s, T z) { return s * digamma_t(z); }
  template <class T> __device__ static T s2(T s, T z) { return s * trigamma_t(z); }
  __device__ static bool rescue(float z) { return !(z > 0.0f); }
};
struct GammaFn {
  template <class T> __device__ static T f0(T z) { return gamma_t(z); }
  // (s·ψ)·Γ: Γψ alone overflows float for z ~ 35 even when s·Γψ does not.
  template <class T> __device__ static T s1(T s, T z) { return (s * digamma_t(z)) * gamma_t(z); }
  template <class T> __device__ static T s2(T s, T z) {
    const T p = digamma_t(z);
    return (s * (p * p + trigamma_t(z))) * gamma_t(z);
  }
  __device__ static bool rescue(float z) { return !(z > 0.0f); }
};
struct DigammaFn {
  template <class T> __device__ static T f0(T z) { return digamma_t(z); }
  template <class T> __device__ static T s1(T s, T z) { return s * trigamma_t(z); }
  template <class T> __device__ static T s2(T s, T z) { return s * tetragamma_t(z); }
  __device__ static bool rescue(float z) { return !(z > 1e-3f); }
};
struct TrigammaFn {
  template <class T> __device__ static T f0(T z) { return trigamma_t(z); }
  template <class T> __device__ static T s1(T s, T z) { return s * tetragamma_t(z); }
  template <class T> __device__ static T s2(T s, T z) { return s * pentagamma_t(z); }
  __device__ static bool rescue(float z) { return !(z > 1e-2f); }
};

template <typename T>
__device__ __forceinline__ bool needs_fp64(bool rescue) {
  return std::is_same<T, float>::value && rescue;
}

// Forward: out = f(z).
template <class F, typename T_>
struct UnaryFwd {
  using T = T_;
  static constexpr int NIN = 1, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    if (needs_fp64<T>(F::rescue((float)in[0]))) out[0] = (T)F::f0((double)in[0]);
    else out[0] = F::f0(in[0]);
  }
};

// Backward: in = {grad, z}, out = grad * f'(z).
template <class F, typename T_>
struct UnaryBwd {
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    if (needs_fp64<T>(F::rescue((float)in[1]))) out[0] = (T)F::s1((double)in[0], (double)in[1]);
    else out[0] = F::s1(in[0], in[1]);
  }
};

// Double backward: in = {gg, grad, z}, out = {gg * f'(z), gg * grad * f''(z)}.
template <class F, typename T_>
struct UnaryBwdBwd {
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = 1;
  static constexpr bool REDUCE = true;
  __device__ static void eval(int, const T* in, T* out, uint32_t mask) {
    if (needs_fp64<T>(F::rescue((float)in[2]))) {
      const double gg = in[0], g = in[1], z = in[2];
      out[0] = (mask & 1u) ? (T)F::s1(gg, z) : T(0);
      out[1] = (mask & 2u) ? (T)F::s2(gg * g, z) : T(0);
    } else {
      out[0] = (mask & 1u) ? F::s1(in[0], in[2]) : T(0);
      out[1] = (mask & 2u) ? F::s2(in[0] * in[1], in[2]) : T(0);
    }
  }
};

#define TSB_UNARY_ALIASES(Name, Fn)                                   \
  template <typename T> using Name##Fwd = UnaryFwd<Fn, T>;           \
  template <typename T> using Name##Bwd = UnaryBwd<Fn, T>;           \
  template <typename T> using Name##BwdBwd = UnaryBwdBwd<Fn, T>;

TSB_UNARY_ALIASES(LogGamma, LogGammaFn)
TSB_UNARY_ALIASES(Gamma, GammaFn)
TSB_UNARY_ALIASES(Digamma, DigammaFn)
TSB_UNARY_ALIASES(Trigamma, TrigammaFn)

}  // namespace tsb

// ------------------------------------------------------------ complex data
// complex64 / complex128 (evaluated in complex128, complex_gamma.cuh).  The
// backward ops return PyTorch's conjugate Wirtinger gradients of these
// holomorphic functions: g·conj(f'(z)); the double backward returns, for the
// backward B(g, z) = g·conj(f'(z)), the gradient in g, gg·f'(z), and in z,
// conj(gg)·g·conj(f''(z)).  (The reference conjugates in gamma_backward.h:19-22
// but not in log_gamma_backward.h or digamma_backward.h, and skips its complex
// gradchecks; here every op follows the convention, so gradcheck holds.)
#include "complex_gamma.cuh"

namespace tsb {

struct CLogGammaFn {
  __device__ static cdouble f0(cdouble z) { return loggamma_c(z); }
  __device__ static cdouble d1(cdouble z) { return digamma_c(z); }
  __device__ static cdouble d2(cdouble z) { return trigamma_c(z); }
};
struct CGammaFn {
  __device__ static cdouble f0(cdouble z) { return gamma_c(z); }
  __device__ static cdouble d1(cdouble z) { return gamma_c(z) * digamma_c(z); }
  __device__ static cdouble d2(cdouble z) {
    const cdouble p = digamma_c(z);
    return gamma_c(z) * (p * p + trigamma_c(z));
  }
};
struct CDigammaFn {
  __device__ static cdouble f0(cdouble z) { return digamma_c(z); }
  __device__ static cdouble d1(cdouble z) { return trigamma_c(z); }
  __device__ static cdouble d2(cdouble z) { return tetragamma_c(z); }
};
struct CTrigammaFn {
  __device__ static cdouble f0(cdouble z) { return trigamma_c(z); }
  __device__ static cdouble d1(cdouble z) { return tetragamma_c(z); }
  __device__ static cdouble d2(cdouble z) { return pentagamma_c(z); }
};

template <class F>
struct CUnaryFwd {
  using T = cdouble;
  static constexpr int NIN = 1, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) { out[0] = F::f0(in[0]); }
};
template <class F>
struct CUnaryBwd {
  using T = cdouble;
  static constexpr int NIN = 2, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) { out[0] = in[0] * cuda::std::conj(F::d1(in[1])); }
};
template <class F>
struct CUnaryBwdBwd {
  using T = cdouble;
  static constexpr int NIN = 3, NOUT = 2, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t mask) {
    if (mask & 1u) out[0] = in[0] * F::d1(in[2]);
    if (mask & 2u) out[1] = cuda::std::conj(in[0]) * in[1] * cuda::std::conj(F::d2(in[2]));
  }
};

}  // namespace tsb
