// Gamma-family entry points (bwd); one translation unit per pass keeps builds parallel.
#include "gamma_ops.cuh"

TSB_DEFINE_OP_C(tsb_log_gamma_backward, tsb::LogGammaBwd, tsb::CUnaryBwd<tsb::CLogGammaFn>)
TSB_DEFINE_OP_C(tsb_gamma_backward, tsb::GammaBwd, tsb::CUnaryBwd<tsb::CGammaFn>)
TSB_DEFINE_OP_C(tsb_digamma_backward, tsb::DigammaBwd, tsb::CUnaryBwd<tsb::CDigammaFn>)
TSB_DEFINE_OP_C(tsb_trigamma_backward, tsb::TrigammaBwd, tsb::CUnaryBwd<tsb::CTrigammaFn>)
