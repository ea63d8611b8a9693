// Gamma, chi-squared and Poisson cumulative distributions (fwd).
#include "probability_ops.cuh"

TSB_DEFINE_OP(tsb_gamma_cumulative_distribution, tsb::GammaCdfFwd)
TSB_DEFINE_OP(tsb_chi2_cumulative_distribution, tsb::Chi2CdfFwd)
TSB_DEFINE_OP(tsb_poisson_cumulative_distribution, tsb::PoissonCdfFwd)
