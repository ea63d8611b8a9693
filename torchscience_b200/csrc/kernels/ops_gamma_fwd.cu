// Gamma-family entry points (fwd); one translation unit per pass keeps builds parallel.
#include "gamma_ops.cuh"

TSB_DEFINE_OP(tsb_log_gamma, tsb::LogGammaFwd)
TSB_DEFINE_OP(tsb_gamma, tsb::GammaFwd)
TSB_DEFINE_OP(tsb_digamma, tsb::DigammaFwd)
TSB_DEFINE_OP(tsb_trigamma, tsb::TrigammaFwd)
