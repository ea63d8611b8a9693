// polygamma (fwd, bwd, double bwd).
#include "beta_ops.cuh"

TSB_DEFINE_OP(tsb_polygamma, tsb::PolygammaFwd)
TSB_DEFINE_OP(tsb_polygamma_backward, tsb::PolygammaBwd)
TSB_DEFINE_OP(tsb_polygamma_backward_backward, tsb::PolygammaBwdBwd)
