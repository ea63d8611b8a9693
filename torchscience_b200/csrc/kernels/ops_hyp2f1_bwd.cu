// Gauss hypergeometric 2F1 entry point (bwd); one translation unit per pass keeps builds parallel.
#include "hyp2f1_ops.cuh"

TSB_DEFINE_OP(tsb_hypergeometric_2_f_1_backward, tsb::Hyp2f1Bwd)
