// lnΓ, Γ, ψ, ψ' — forward, backward and double-backward entry points.
// Reference scalar kernels: log_gamma.h, gamma.h, digamma.h, trigamma.h and
// their *_backward / *_backward_backward headers (same formulas:
// d lnΓ = ψ, dΓ = Γψ, d²Γ = Γ(ψ² + ψ'), dψ = ψ', dψ' = ψ'').
#include "dispatch.cuh"
#include "gamma_math.cuh"

namespace tsb {

template <typename T>
__device__ __forceinline__ T gamma_deriv1(T z) {
  return gamma_t(z) * digamma_t(z);
}
template <typename T>
__device__ __forceinline__ T gamma_deriv2(T z) {
  const T p = digamma_t(z);
  return gamma_t(z) * (p * p + trigamma_t(z));
}

#define TSB_UNARY_FUNCTORS(Name, F0, F1, F2)                                          \
  template <typename T_>                                                              \
  struct Name##Fwd {                                                                  \
    using T = T_;                                                                     \
    static constexpr int NIN = 1, NOUT = 1, R = 1;                                    \
    static constexpr bool REDUCE = false;                                             \
    __device__ static void eval(int, const T* in, T* out, uint32_t) { out[0] = F0(in[0]); } \
  };                                                                                  \
  template <typename T_>                                                              \
  struct Name##Bwd {                                                                  \
    using T = T_;                                                                     \
    static constexpr int NIN = 2, NOUT = 1, R = 1;                                    \
    static constexpr bool REDUCE = false;                                             \
    __device__ static void eval(int, const T* in, T* out, uint32_t) { out[0] = in[0] * F1(in[1]); } \
  };                                                                                  \
  template <typename T_>                                                              \
  struct Name##BwdBwd {                                                               \
    using T = T_;                                                                     \
    static constexpr int NIN = 3, NOUT = 2, R = 1;                                    \
    static constexpr bool REDUCE = true;                                              \
    __device__ static void eval(int, const T* in, T* out, uint32_t mask) {            \
      out[0] = (mask & 1u) ? in[0] * F1(in[2]) : T(0);                                \
      out[1] = (mask & 2u) ? in[0] * in[1] * F2(in[2]) : T(0);                        \
    }                                                                                 \
  };

TSB_UNARY_FUNCTORS(LogGamma, lgamma_t, digamma_t, trigamma_t)
TSB_UNARY_FUNCTORS(Gamma, gamma_t, gamma_deriv1, gamma_deriv2)
TSB_UNARY_FUNCTORS(Digamma, digamma_t, trigamma_t, tetragamma_t)
TSB_UNARY_FUNCTORS(Trigamma, trigamma_t, tetragamma_t, pentagamma_t)

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
