// Incomplete gamma entry points (bwd); one translation unit per pass keeps builds parallel.
#include "igamma_ops.cuh"

TSB_DEFINE_OP(tsb_regularized_gamma_p_backward, tsb::GammaPBwd)
TSB_DEFINE_OP(tsb_regularized_gamma_q_backward, tsb::GammaQBwd)
