// lnΓ, Γ, ψ, ψ' — forward, backward and double-backward entry points.
// Reference scalar kernels: log_gamma.h, gamma.h, digamma.h, trigamma.h and
// their *_backward / *_backward_backward headers (same formulas:
// d lnΓ = ψ, dΓ = Γψ, d²Γ = Γ(ψ² + ψ'), dψ = ψ', dψ' = ψ'').
//
// FP64 kernels (double data) evaluate everything in double with one region.
// Mixed kernels (float/half/bf16 data) classify each element into region 0
// (FP32 evaluation) or region 1 (FP64 evaluation of the same formula, for
// arguments the FP32 path would not hold to 1e-6); the map kernel's
// compaction keeps the two paths in separate warps.
#include <type_traits>

#include "dispatch.cuh"
#include "gamma_math.cuh"

namespace tsb {

struct LogGammaFn {
  template <class T> __device__ static T f0(T z) { return lgamma_t(z); }
  template <class T> __device__ static T f1(T z) { return digamma_t(z); }
  template <class T> __device__ static T f2(T z) { return trigamma_t(z); }
  // lnΓ cancels near its zeros at 1 and 2; x <= 0 uses reflection.
  __device__ static bool rescue(float z) { return !(z > 0.0f) || (z > 0.5f && z < 3.0f); }
};
struct GammaFn {
  template <class T> __device__ static T f0(T z) { return gamma_t(z); }
  template <class T> __device__ static T f1(T z) { return gamma_t(z) * digamma_t(z); }
  template <class T> __device__ static T f2(T z) {
    const T p = digamma_t(z);
    return gamma_t(z) * (p * p + trigamma_t(z));
  }
  // Γψ and Γ(ψ²+ψ') overflow float before the upstream gradient scales them.
  __device__ static bool rescue(float z) { return !(z > 0.0f) || z > 30.0f; }
};
struct DigammaFn {
  template <class T> __device__ static T f0(T z) { return digamma_t(z); }
  template <class T> __device__ static T f1(T z) { return trigamma_t(z); }
  template <class T> __device__ static T f2(T z) { return tetragamma_t(z); }
  __device__ static bool rescue(float z) { return !(z > 1e-3f); }
};
struct TrigammaFn {
  template <class T> __device__ static T f0(T z) { return trigamma_t(z); }
  template <class T> __device__ static T f1(T z) { return tetragamma_t(z); }
  template <class T> __device__ static T f2(T z) { return pentagamma_t(z); }
  __device__ static bool rescue(float z) { return !(z > 1e-2f); }
};

template <typename T>
constexpr int kMixedRegions = std::is_same<T, float>::value ? 2 : 1;

// Forward: out = f(z).
template <class F, typename T_>
struct UnaryFwd {
  using T = T_;
  static constexpr int NIN = 1, NOUT = 1, R = kMixedRegions<T_>;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) { return F::rescue((float)in[0]) ? 1 : 0; }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) {
    if (R == 2 && r == 1) out[0] = (T)F::f0((double)in[0]);
    else out[0] = F::f0(in[0]);
  }
};

// Backward: in = {grad, z}, out = grad * f'(z).
template <class F, typename T_>
struct UnaryBwd {
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = kMixedRegions<T_>;
  static constexpr bool REDUCE = false;
  __device__ static int classify(const T* in) { return F::rescue((float)in[1]) ? 1 : 0; }
  __device__ static void eval(int r, const T* in, T* out, uint32_t) {
    if (R == 2 && r == 1) out[0] = (T)((double)in[0] * F::f1((double)in[1]));
    else out[0] = in[0] * F::f1(in[1]);
  }
};

// Double backward: in = {gg, grad, z}, out = {gg * f'(z), gg * grad * f''(z)}.
template <class F, typename T_>
struct UnaryBwdBwd {
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = kMixedRegions<T_>;
  static constexpr bool REDUCE = true;
  __device__ static int classify(const T* in) { return F::rescue((float)in[2]) ? 1 : 0; }
  __device__ static void eval(int r, const T* in, T* out, uint32_t mask) {
    if (R == 2 && r == 1) {
      const double gg = in[0], g = in[1], z = in[2];
      out[0] = (mask & 1u) ? (T)(gg * F::f1(z)) : T(0);
      out[1] = (mask & 2u) ? (T)(gg * g * F::f2(z)) : T(0);
    } else {
      out[0] = (mask & 1u) ? in[0] * F::f1(in[2]) : T(0);
      out[1] = (mask & 2u) ? in[0] * in[1] * F::f2(in[2]) : T(0);
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

TSB_DEFINE_OP(tsb_log_gamma, tsb::LogGammaFwd)
TSB_DEFINE_OP(tsb_log_gamma_backward, tsb::LogGammaBwd)
TSB_DEFINE_OP(tsb_log_gamma_backward_backward, tsb::LogGammaBwdBwd)
TSB_DEFINE_OP(tsb_gamma, tsb::GammaFwd)
TSB_DEFINE_OP(tsb_gamma_backward, tsb::GammaBwd)
TSB_DEFINE_OP(tsb_gamma_backward_backward, tsb::GammaBwdBwd)
TSB_DEFINE_OP(tsb_digamma, tsb::DigammaFwd)
TSB_DEFINE_OP(tsb_digamma_backward, tsb::DigammaBwd)
TSB_DEFINE_OP(tsb_digamma_backward_backward, tsb::DigammaBwdBwd)
TSB_DEFINE_OP(tsb_trigamma, tsb::TrigammaFwd)
TSB_DEFINE_OP(tsb_trigamma_backward, tsb::TrigammaBwd)
TSB_DEFINE_OP(tsb_trigamma_backward_backward, tsb::TrigammaBwdBwd)
