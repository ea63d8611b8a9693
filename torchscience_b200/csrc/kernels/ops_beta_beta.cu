// beta (fwd, bwd, double bwd).
#include "beta_ops.cuh"

TSB_DEFINE_OP(tsb_beta, tsb::BetaFwd)
TSB_DEFINE_OP(tsb_beta_backward, tsb::BetaBwd)
TSB_DEFINE_OP(tsb_beta_backward_backward, tsb::BetaBwdBwd)
