// Integer-order Bessel functions as unary ops (fwd).
#include "bessel_ops.cuh"

TSB_DEFINE_OP(tsb_bessel_j_1, tsb::BesselJ1Fwd)
TSB_DEFINE_OP(tsb_bessel_y_0, tsb::BesselY0Fwd)
TSB_DEFINE_OP(tsb_bessel_y_1, tsb::BesselY1Fwd)
TSB_DEFINE_OP(tsb_modified_bessel_i_0, tsb::ModifiedBesselI0Fwd)
TSB_DEFINE_OP(tsb_modified_bessel_i_1, tsb::ModifiedBesselI1Fwd)
TSB_DEFINE_OP(tsb_modified_bessel_k_0, tsb::ModifiedBesselK0Fwd)
TSB_DEFINE_OP(tsb_modified_bessel_k_1, tsb::ModifiedBesselK1Fwd)
