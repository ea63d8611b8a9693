// Spherical Bessel j_n of real order (fwd, bwd, double bwd).
#include "spherical_ops.cuh"

TSB_DEFINE_OP(tsb_spherical_bessel_j, tsb::SphJFwd)
TSB_DEFINE_OP(tsb_spherical_bessel_j_backward, tsb::SphJBwd)
TSB_DEFINE_OP(tsb_spherical_bessel_j_backward_backward, tsb::SphJBwdBwd)
