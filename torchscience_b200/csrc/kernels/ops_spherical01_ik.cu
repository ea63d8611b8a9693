// Modified spherical Bessel i and k of order 0 and 1 as unary ops (fwd, bwd, double bwd).
#include "spherical_ops.cuh"

TSB_DEFINE_OP(tsb_spherical_bessel_i_0, tsb::SphI0Fwd)
TSB_DEFINE_OP(tsb_spherical_bessel_i_0_backward, tsb::SphI0Bwd)
TSB_DEFINE_OP(tsb_spherical_bessel_i_0_backward_backward, tsb::SphI0BwdBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_i_1, tsb::SphI1Fwd)
TSB_DEFINE_OP(tsb_spherical_bessel_i_1_backward, tsb::SphI1Bwd)
TSB_DEFINE_OP(tsb_spherical_bessel_i_1_backward_backward, tsb::SphI1BwdBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_k_0, tsb::SphK0Fwd)
TSB_DEFINE_OP(tsb_spherical_bessel_k_0_backward, tsb::SphK0Bwd)
TSB_DEFINE_OP(tsb_spherical_bessel_k_0_backward_backward, tsb::SphK0BwdBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_k_1, tsb::SphK1Fwd)
TSB_DEFINE_OP(tsb_spherical_bessel_k_1_backward, tsb::SphK1Bwd)
TSB_DEFINE_OP(tsb_spherical_bessel_k_1_backward_backward, tsb::SphK1BwdBwd)
