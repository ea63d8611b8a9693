// Modified spherical Bessel k_n of real order (fwd, bwd, double bwd).
#include "spherical_ops.cuh"

TSB_DEFINE_OP(tsb_spherical_bessel_k, tsb::SphKFwd)
TSB_DEFINE_OP(tsb_spherical_bessel_k_backward, tsb::SphKBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_k_backward_backward, tsb::SphKBwdBwd)
