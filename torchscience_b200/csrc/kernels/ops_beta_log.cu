// log_beta (fwd, bwd, double bwd).
#include "beta_ops.cuh"

TSB_DEFINE_OP(tsb_log_beta, tsb::LogBetaFwd)
TSB_DEFINE_OP(tsb_log_beta_backward, tsb::LogBetaBwd)
TSB_DEFINE_OP(tsb_log_beta_backward_backward, tsb::LogBetaBwdBwd)
