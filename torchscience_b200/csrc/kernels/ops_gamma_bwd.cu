// Gamma-family entry points (bwd); one translation unit per pass keeps builds parallel.
#include "gamma_ops.cuh"

TSB_DEFINE_OP(tsb_log_gamma_backward, tsb::LogGammaBwd)
TSB_DEFINE_OP(tsb_gamma_backward, tsb::GammaBwd)
TSB_DEFINE_OP(tsb_digamma_backward, tsb::DigammaBwd)
TSB_DEFINE_OP(tsb_trigamma_backward, tsb::TrigammaBwd)
