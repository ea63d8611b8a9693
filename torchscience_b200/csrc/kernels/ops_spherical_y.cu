// Spherical Bessel y_n of real order (fwd, bwd, double bwd).
#include "spherical_ops.cuh"

TSB_DEFINE_OP(tsb_spherical_bessel_y, tsb::SphYFwd)
TSB_DEFINE_OP(tsb_spherical_bessel_y_backward, tsb::SphYBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_y_backward_backward, tsb::SphYBwdBwd)
