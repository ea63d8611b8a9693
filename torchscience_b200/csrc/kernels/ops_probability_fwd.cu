// Probability callers of the incomplete gamma: cumulative distributions, the χ² survival function and the gamma and χ² densities (fwd).
#include "probability_ops.cuh"

TSB_DEFINE_OP(tsb_gamma_cumulative_distribution, tsb::GammaCdfFwd)
TSB_DEFINE_OP(tsb_chi2_cumulative_distribution, tsb::Chi2CdfFwd)
TSB_DEFINE_OP(tsb_poisson_cumulative_distribution, tsb::PoissonCdfFwd)
TSB_DEFINE_OP(tsb_chi2_survival, tsb::Chi2SurvivalFwd)
TSB_DEFINE_OP(tsb_gamma_probability_density, tsb::GammaPdfFwd)
TSB_DEFINE_OP(tsb_chi2_probability_density, tsb::Chi2PdfFwd)
