// Gamma-family entry points (fwd); one translation unit per pass keeps builds parallel.
#include "gamma_ops.cuh"

TSB_DEFINE_OP_C(tsb_log_gamma, tsb::LogGammaFwd, tsb::CUnaryFwd<tsb::CLogGammaFn>)
TSB_DEFINE_OP_C(tsb_gamma, tsb::GammaFwd, tsb::CUnaryFwd<tsb::CGammaFn>)
TSB_DEFINE_OP_C(tsb_digamma, tsb::DigammaFwd, tsb::CUnaryFwd<tsb::CDigammaFn>)
TSB_DEFINE_OP_C(tsb_trigamma, tsb::TrigammaFwd, tsb::CUnaryFwd<tsb::CTrigammaFn>)
