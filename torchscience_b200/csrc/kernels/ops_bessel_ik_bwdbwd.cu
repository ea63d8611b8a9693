// Modified Bessel I_ν, K_ν entry points (bwdbwd); one translation unit per pass keeps builds parallel.
#include "bessel_ops.cuh"

TSB_DEFINE_OP(tsb_modified_bessel_i_backward_backward, tsb::BesselIBwdBwd)
TSB_DEFINE_OP(tsb_modified_bessel_k_backward_backward, tsb::BesselKBwdBwd)
