// Incomplete gamma forward with first derivatives (autograd's forward when
// an input requires grad) and the backward from kept derivatives.
#include "igamma_ops.cuh"

TSB_DEFINE_OP(tsb_regularized_gamma_p_forward_with_grads, tsb::GammaPFwdGrad)
TSB_DEFINE_OP(tsb_regularized_gamma_q_forward_with_grads, tsb::GammaQFwdGrad)
TSB_DEFINE_OP(tsb_gradient_product, tsb::GradProductD)
