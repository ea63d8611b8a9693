// incomplete_beta (fwd, bwd, double bwd).
#include "ibeta_ops.cuh"

TSB_DEFINE_OP(tsb_incomplete_beta, tsb::IbetaFwd)
TSB_DEFINE_OP(tsb_incomplete_beta_backward, tsb::IbetaBwd)
TSB_DEFINE_OP(tsb_incomplete_beta_backward_backward, tsb::IbetaBwdBwd)
