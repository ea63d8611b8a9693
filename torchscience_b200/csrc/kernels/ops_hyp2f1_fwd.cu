// Gauss hypergeometric 2F1 entry point (fwd); one translation unit per pass keeps builds parallel.
#include "hyp2f1_ops.cuh"

TSB_DEFINE_OP(tsb_hypergeometric_2_f_1, tsb::Hyp2f1Fwd)
