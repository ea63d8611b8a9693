// Spherical Bessel functions of real order (fwd, bwd, double bwd).
#include "spherical_ops.cuh"

TSB_DEFINE_OP(tsb_spherical_bessel_j, tsb::SphJFwd)
TSB_DEFINE_OP(tsb_spherical_bessel_j_backward, tsb::SphJBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_j_backward_backward, tsb::SphJBwdBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_y, tsb::SphYFwd)
TSB_DEFINE_OP(tsb_spherical_bessel_y_backward, tsb::SphYBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_y_backward_backward, tsb::SphYBwdBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_i, tsb::SphIFwd)
TSB_DEFINE_OP(tsb_spherical_bessel_i_backward, tsb::SphIBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_i_backward_backward, tsb::SphIBwdBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_k, tsb::SphKFwd)
TSB_DEFINE_OP(tsb_spherical_bessel_k_backward, tsb::SphKBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_k_backward_backward, tsb::SphKBwdBwd)
