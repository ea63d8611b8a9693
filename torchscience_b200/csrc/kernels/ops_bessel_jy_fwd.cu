// Bessel J_ν, Y_ν and J_0 entry points (fwd); one translation unit per pass keeps builds parallel.
#include "bessel_ops.cuh"

TSB_DEFINE_OP(tsb_bessel_j, tsb::BesselJFwd)
TSB_DEFINE_OP(tsb_bessel_y, tsb::BesselYFwd)
TSB_DEFINE_OP(tsb_bessel_j_0, tsb::BesselJ0Fwd)
