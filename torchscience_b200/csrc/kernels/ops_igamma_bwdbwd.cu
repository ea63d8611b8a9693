// Incomplete gamma entry points (bwdbwd); one translation unit per pass keeps builds parallel.
#include "igamma_ops.cuh"

TSB_DEFINE_OP(tsb_regularized_gamma_p_backward_backward, tsb::GammaPBwdBwd)
TSB_DEFINE_OP(tsb_regularized_gamma_q_backward_backward, tsb::GammaQBwdBwd)
