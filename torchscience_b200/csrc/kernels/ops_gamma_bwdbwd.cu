// Gamma-family entry points (bwdbwd); one translation unit per pass keeps builds parallel.
#include "gamma_ops.cuh"

TSB_DEFINE_OP(tsb_log_gamma_backward_backward, tsb::LogGammaBwdBwd)
TSB_DEFINE_OP(tsb_gamma_backward_backward, tsb::GammaBwdBwd)
TSB_DEFINE_OP(tsb_digamma_backward_backward, tsb::DigammaBwdBwd)
TSB_DEFINE_OP(tsb_trigamma_backward_backward, tsb::TrigammaBwdBwd)
