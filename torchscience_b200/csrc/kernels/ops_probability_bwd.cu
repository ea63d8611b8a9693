// Gamma, chi-squared and Poisson cumulative distributions (bwd).
#include "probability_ops.cuh"

TSB_DEFINE_OP(tsb_gamma_cumulative_distribution_backward, tsb::GammaCdfBwd)
TSB_DEFINE_OP(tsb_chi2_cumulative_distribution_backward, tsb::Chi2CdfBwd)
TSB_DEFINE_OP(tsb_poisson_cumulative_distribution_backward, tsb::PoissonCdfBwd)
