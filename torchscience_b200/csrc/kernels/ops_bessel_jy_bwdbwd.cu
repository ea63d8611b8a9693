// Bessel J_ν, Y_ν and J_0 entry points (bwdbwd); one translation unit per pass keeps builds parallel.
#include "bessel_ops.cuh"

TSB_DEFINE_OP(tsb_bessel_j_backward_backward, tsb::BesselJBwdBwd)
TSB_DEFINE_OP(tsb_bessel_y_backward_backward, tsb::BesselYBwdBwd)
TSB_DEFINE_OP(tsb_bessel_j_0_backward_backward, tsb::BesselJ0BwdBwd)
