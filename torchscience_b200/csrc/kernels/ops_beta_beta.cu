// beta (fwd, bwd, double bwd).
#include "beta_ops.cuh"

TSB_DEFINE_OP_C(tsb_beta, tsb::BetaFwd, tsb::CBetaFwd<true>)
TSB_DEFINE_OP_C(tsb_beta_backward, tsb::BetaBwd, tsb::CBetaBwd<true>)
TSB_DEFINE_OP_C(tsb_beta_backward_backward, tsb::BetaBwdBwd, tsb::CBetaBwdBwd<true>)
