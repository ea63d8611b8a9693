// log_beta (fwd, bwd, double bwd).
#include "beta_ops.cuh"

TSB_DEFINE_OP_C(tsb_log_beta, tsb::LogBetaFwd, tsb::CBetaFwd<false>)
TSB_DEFINE_OP_C(tsb_log_beta_backward, tsb::LogBetaBwd, tsb::CBetaBwd<false>)
TSB_DEFINE_OP_C(tsb_log_beta_backward_backward, tsb::LogBetaBwdBwd, tsb::CBetaBwdBwd<false>)
