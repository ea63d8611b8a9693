// Incomplete gamma entry points (fwd); one translation unit per pass keeps builds parallel.
#include "igamma_ops.cuh"

TSB_DEFINE_OP(tsb_regularized_gamma_p, tsb::GammaPFwd)
TSB_DEFINE_OP(tsb_regularized_gamma_q, tsb::GammaQFwd)
