// Bessel J_ν, Y_ν and J_0 entry points (bwd); one translation unit per pass keeps builds parallel.
#include "bessel_ops.cuh"

TSB_DEFINE_OP(tsb_bessel_j_backward, tsb::BesselJBwd)
TSB_DEFINE_OP(tsb_bessel_y_backward, tsb::BesselYBwd)
TSB_DEFINE_OP(tsb_bessel_j_0_backward, tsb::BesselJ0Bwd)
