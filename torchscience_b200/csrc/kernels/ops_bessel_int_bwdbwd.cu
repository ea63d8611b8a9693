// Integer-order Bessel functions as unary ops (bwdbwd).
#include "bessel_ops.cuh"

TSB_DEFINE_OP(tsb_bessel_j_1_backward_backward, tsb::BesselJ1BwdBwd)
TSB_DEFINE_OP(tsb_bessel_y_0_backward_backward, tsb::BesselY0BwdBwd)
TSB_DEFINE_OP(tsb_bessel_y_1_backward_backward, tsb::BesselY1BwdBwd)
TSB_DEFINE_OP(tsb_modified_bessel_i_0_backward_backward, tsb::ModifiedBesselI0BwdBwd)
TSB_DEFINE_OP(tsb_modified_bessel_i_1_backward_backward, tsb::ModifiedBesselI1BwdBwd)
TSB_DEFINE_OP(tsb_modified_bessel_k_0_backward_backward, tsb::ModifiedBesselK0BwdBwd)
TSB_DEFINE_OP(tsb_modified_bessel_k_1_backward_backward, tsb::ModifiedBesselK1BwdBwd)
