// log_beta, beta and polygamma (fwd, bwd, double bwd).
#include "beta_ops.cuh"

TSB_DEFINE_OP(tsb_log_beta, tsb::LogBetaFwd)
TSB_DEFINE_OP(tsb_log_beta_backward, tsb::LogBetaBwd)
TSB_DEFINE_OP(tsb_log_beta_backward_backward, tsb::LogBetaBwdBwd)
TSB_DEFINE_OP(tsb_beta, tsb::BetaFwd)
TSB_DEFINE_OP(tsb_beta_backward, tsb::BetaBwd)
TSB_DEFINE_OP(tsb_beta_backward_backward, tsb::BetaBwdBwd)
TSB_DEFINE_OP(tsb_polygamma, tsb::PolygammaFwd)
TSB_DEFINE_OP(tsb_polygamma_backward, tsb::PolygammaBwd)
TSB_DEFINE_OP(tsb_polygamma_backward_backward, tsb::PolygammaBwdBwd)
