// Gamma-family entry points (bwdbwd); one translation unit per pass keeps builds parallel.
#include "gamma_ops.cuh"

TSB_DEFINE_OP_C(tsb_log_gamma_backward_backward, tsb::LogGammaBwdBwd, tsb::CUnaryBwdBwd<tsb::CLogGammaFn>)
TSB_DEFINE_OP_C(tsb_gamma_backward_backward, tsb::GammaBwdBwd, tsb::CUnaryBwdBwd<tsb::CGammaFn>)
TSB_DEFINE_OP_C(tsb_digamma_backward_backward, tsb::DigammaBwdBwd, tsb::CUnaryBwdBwd<tsb::CDigammaFn>)
TSB_DEFINE_OP_C(tsb_trigamma_backward_backward, tsb::TrigammaBwdBwd, tsb::CUnaryBwdBwd<tsb::CTrigammaFn>)
