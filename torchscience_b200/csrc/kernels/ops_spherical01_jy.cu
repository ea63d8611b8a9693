// Spherical Bessel j and y of order 0 and 1 as unary ops (fwd, bwd, double bwd).
#include "spherical_ops.cuh"

TSB_DEFINE_OP(tsb_spherical_bessel_j_0, tsb::SphJ0Fwd)
TSB_DEFINE_OP(tsb_spherical_bessel_j_0_backward, tsb::SphJ0Bwd)
TSB_DEFINE_OP(tsb_spherical_bessel_j_0_backward_backward, tsb::SphJ0BwdBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_j_1, tsb::SphJ1Fwd)
TSB_DEFINE_OP(tsb_spherical_bessel_j_1_backward, tsb::SphJ1Bwd)
TSB_DEFINE_OP(tsb_spherical_bessel_j_1_backward_backward, tsb::SphJ1BwdBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_y_0, tsb::SphY0Fwd)
TSB_DEFINE_OP(tsb_spherical_bessel_y_0_backward, tsb::SphY0Bwd)
TSB_DEFINE_OP(tsb_spherical_bessel_y_0_backward_backward, tsb::SphY0BwdBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_y_1, tsb::SphY1Fwd)
TSB_DEFINE_OP(tsb_spherical_bessel_y_1_backward, tsb::SphY1Bwd)
TSB_DEFINE_OP(tsb_spherical_bessel_y_1_backward_backward, tsb::SphY1BwdBwd)
