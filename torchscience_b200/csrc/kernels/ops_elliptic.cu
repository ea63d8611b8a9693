// Complete elliptic integrals K(m), E(m): forward, backward and
// double-backward entry points (dK/dm, dE/dm and second derivatives are
// analytic, see elliptic_math.cuh).
#include "dispatch.cuh"
#include "elliptic_math.cuh"

namespace tsb {

template <typename T_, bool SECOND_KIND>
struct EllipFwd {
  using T = T_;
  static constexpr int NIN = 1, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const EllipKE<T> r = ellip_t<0>(in[0]);
    out[0] = SECOND_KIND ? r.E : r.K;
  }
};

template <typename T_, bool SECOND_KIND>
struct EllipBwd {
  using T = T_;
  static constexpr int NIN = 2, NOUT = 1, R = 1;
  static constexpr bool REDUCE = false;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const EllipKE<T> r = ellip_t<1>(in[1]);
    out[0] = in[0] * (SECOND_KIND ? r.Ep : r.Kp);
  }
};

template <typename T_, bool SECOND_KIND>
struct EllipBwdBwd {
  using T = T_;
  static constexpr int NIN = 3, NOUT = 2, R = 1;
  static constexpr bool REDUCE = true;
  __device__ static void eval(int, const T* in, T* out, uint32_t) {
    const EllipKE<T> r = ellip_t<2>(in[2]);
    out[0] = in[0] * (SECOND_KIND ? r.Ep : r.Kp);
    out[1] = in[0] * in[1] * (SECOND_KIND ? r.Epp : r.Kpp);
  }
};

template <typename T> using EllipKFwd = EllipFwd<T, false>;
template <typename T> using EllipKBwd = EllipBwd<T, false>;
template <typename T> using EllipKBwdBwd = EllipBwdBwd<T, false>;
template <typename T> using EllipEFwd = EllipFwd<T, true>;
template <typename T> using EllipEBwd = EllipBwd<T, true>;
template <typename T> using EllipEBwdBwd = EllipBwdBwd<T, true>;

}  // namespace tsb

TSB_DEFINE_OP(tsb_complete_legendre_elliptic_integral_k, tsb::EllipKFwd)
TSB_DEFINE_OP(tsb_complete_legendre_elliptic_integral_k_backward, tsb::EllipKBwd)
TSB_DEFINE_OP(tsb_complete_legendre_elliptic_integral_k_backward_backward, tsb::EllipKBwdBwd)
TSB_DEFINE_OP(tsb_complete_legendre_elliptic_integral_e, tsb::EllipEFwd)
TSB_DEFINE_OP(tsb_complete_legendre_elliptic_integral_e_backward, tsb::EllipEBwd)
TSB_DEFINE_OP(tsb_complete_legendre_elliptic_integral_e_backward_backward, tsb::EllipEBwdBwd)
