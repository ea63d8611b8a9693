// Probability callers of the incomplete gamma: cumulative distributions, the χ² survival function and the gamma and χ² densities (bwd).
#include "probability_ops.cuh"

TSB_DEFINE_OP(tsb_gamma_cumulative_distribution_backward, tsb::GammaCdfBwd)
TSB_DEFINE_OP(tsb_chi2_cumulative_distribution_backward, tsb::Chi2CdfBwd)
TSB_DEFINE_OP(tsb_poisson_cumulative_distribution_backward, tsb::PoissonCdfBwd)
TSB_DEFINE_OP(tsb_chi2_survival_backward, tsb::Chi2SurvivalBwd)
TSB_DEFINE_OP(tsb_gamma_probability_density_backward, tsb::GammaPdfBwd)
TSB_DEFINE_OP(tsb_chi2_probability_density_backward, tsb::Chi2PdfBwd)
