// Modified spherical Bessel i_n of real order (fwd, bwd, double bwd).
#include "spherical_ops.cuh"

TSB_DEFINE_OP(tsb_spherical_bessel_i, tsb::SphIFwd)
TSB_DEFINE_OP(tsb_spherical_bessel_i_backward, tsb::SphIBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_i_backward_backward, tsb::SphIBwdBwd)
