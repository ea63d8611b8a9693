// Integer-order Bessel functions as unary ops (bwd).
#include "bessel_ops.cuh"

TSB_DEFINE_OP(tsb_bessel_j_1_backward, tsb::BesselJ1Bwd)
TSB_DEFINE_OP(tsb_bessel_y_0_backward, tsb::BesselY0Bwd)
TSB_DEFINE_OP(tsb_bessel_y_1_backward, tsb::BesselY1Bwd)
TSB_DEFINE_OP(tsb_modified_bessel_i_0_backward, tsb::ModifiedBesselI0Bwd)
TSB_DEFINE_OP(tsb_modified_bessel_i_1_backward, tsb::ModifiedBesselI1Bwd)
TSB_DEFINE_OP(tsb_modified_bessel_k_0_backward, tsb::ModifiedBesselK0Bwd)
TSB_DEFINE_OP(tsb_modified_bessel_k_1_backward, tsb::ModifiedBesselK1Bwd)
