// Modified Bessel I_ν, K_ν entry points (fwd); one translation unit per pass keeps builds parallel.
#include "bessel_ops.cuh"

TSB_DEFINE_OP(tsb_modified_bessel_i, tsb::BesselIFwd)
TSB_DEFINE_OP(tsb_modified_bessel_k, tsb::BesselKFwd)
