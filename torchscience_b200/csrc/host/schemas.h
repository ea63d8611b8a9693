// Schema strings of the special-function operators on the accelerated path,
// identical to the reference's TORCH_LIBRARY(torchscience, ...) block in
// src/torchscience/csrc/torchscience.cpp (line numbers per group below).
// Shared by this package's registration and by the oracle's build of the
// reference's CPU operators, so both expose the same torch.ops.torchscience
// interface.
#pragma once

#define TSB_DEFINE_TORCHSCIENCE_SCHEMAS(m)                                                                          \
  /* torchscience.cpp:813-815 */                                                                                     \
  (m).def("gamma(Tensor z) -> Tensor");                                                                              \
  (m).def("gamma_backward(Tensor grad_output, Tensor z) -> Tensor");                                                 \
  (m).def("gamma_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");                 \
  /* torchscience.cpp:817-819 */                                                                                     \
  (m).def("digamma(Tensor z) -> Tensor");                                                                            \
  (m).def("digamma_backward(Tensor grad_output, Tensor z) -> Tensor");                                               \
  (m).def("digamma_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");               \
  /* torchscience.cpp:821-823 */                                                                                     \
  (m).def("trigamma(Tensor z) -> Tensor");                                                                           \
  (m).def("trigamma_backward(Tensor grad_output, Tensor z) -> Tensor");                                              \
  (m).def("trigamma_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");              \
  /* torchscience.cpp:825-827 */                                                                                     \
  (m).def("beta(Tensor a, Tensor b) -> Tensor");                                                                     \
  (m).def("beta_backward(Tensor grad_output, Tensor a, Tensor b) -> (Tensor, Tensor)");                              \
  (m).def(                                                                                                           \
      "beta_backward_backward(Tensor gg_a, Tensor gg_b, Tensor grad_output, Tensor a, Tensor b) -> (Tensor, Tensor, " \
      "Tensor)");                                                                                                    \
  /* torchscience.cpp:841-843 */                                                                                     \
  (m).def("polygamma(Tensor n, Tensor z) -> Tensor");                                                                \
  (m).def("polygamma_backward(Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor)");                         \
  (m).def(                                                                                                           \
      "polygamma_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> (Tensor, "    \
      "Tensor, Tensor)");                                                                                            \
  /* torchscience.cpp:845-847 */                                                                                     \
  (m).def("log_beta(Tensor a, Tensor b) -> Tensor");                                                                 \
  (m).def("log_beta_backward(Tensor grad_output, Tensor a, Tensor b) -> (Tensor, Tensor)");                          \
  (m).def(                                                                                                           \
      "log_beta_backward_backward(Tensor gg_a, Tensor gg_b, Tensor grad_output, Tensor a, Tensor b) -> (Tensor, "     \
      "Tensor, Tensor)");                                                                                            \
  /* torchscience.cpp:877-879 */                                                                                       \
  (m).def("bessel_j_1(Tensor z) -> Tensor");                                                                           \
  (m).def("bessel_j_1_backward(Tensor grad_output, Tensor z) -> Tensor");                                              \
  (m).def("bessel_j_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");              \
  /* torchscience.cpp:882-884 */                                                                                       \
  (m).def("bessel_y_0(Tensor z) -> Tensor");                                                                           \
  (m).def("bessel_y_0_backward(Tensor grad_output, Tensor z) -> Tensor");                                              \
  (m).def("bessel_y_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");              \
  /* torchscience.cpp:887-889 */                                                                                       \
  (m).def("bessel_y_1(Tensor z) -> Tensor");                                                                           \
  (m).def("bessel_y_1_backward(Tensor grad_output, Tensor z) -> Tensor");                                              \
  (m).def("bessel_y_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");              \
  /* torchscience.cpp:862-864 */                                                                                       \
  (m).def("modified_bessel_i_0(Tensor z) -> Tensor");                                                                  \
  (m).def("modified_bessel_i_0_backward(Tensor grad_output, Tensor z) -> Tensor");                                     \
  (m).def("modified_bessel_i_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");     \
  /* torchscience.cpp:867-869 */                                                                                       \
  (m).def("modified_bessel_i_1(Tensor z) -> Tensor");                                                                  \
  (m).def("modified_bessel_i_1_backward(Tensor grad_output, Tensor z) -> Tensor");                                     \
  (m).def("modified_bessel_i_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");     \
  /* torchscience.cpp:892-894 */                                                                                       \
  (m).def("modified_bessel_k_0(Tensor z) -> Tensor");                                                                  \
  (m).def("modified_bessel_k_0_backward(Tensor grad_output, Tensor z) -> Tensor");                                     \
  (m).def("modified_bessel_k_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");     \
  /* torchscience.cpp:897-899 */                                                                                       \
  (m).def("modified_bessel_k_1(Tensor z) -> Tensor");                                                                  \
  (m).def("modified_bessel_k_1_backward(Tensor grad_output, Tensor z) -> Tensor");                                     \
  (m).def("modified_bessel_k_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");     \
  /* torchscience.cpp:922-924 */                                                                                       \
  (m).def("spherical_bessel_j_0(Tensor z) -> Tensor");                                                                 \
  (m).def("spherical_bessel_j_0_backward(Tensor grad_output, Tensor z) -> Tensor");                                    \
  (m).def("spherical_bessel_j_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");    \
  /* torchscience.cpp:927-929 */                                                                                       \
  (m).def("spherical_bessel_j_1(Tensor z) -> Tensor");                                                                 \
  (m).def("spherical_bessel_j_1_backward(Tensor grad_output, Tensor z) -> Tensor");                                    \
  (m).def("spherical_bessel_j_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");    \
  /* torchscience.cpp:937-939 */                                                                                       \
  (m).def("spherical_bessel_y_0(Tensor z) -> Tensor");                                                                 \
  (m).def("spherical_bessel_y_0_backward(Tensor grad_output, Tensor z) -> Tensor");                                    \
  (m).def("spherical_bessel_y_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");    \
  /* torchscience.cpp:942-944 */                                                                                       \
  (m).def("spherical_bessel_y_1(Tensor z) -> Tensor");                                                                 \
  (m).def("spherical_bessel_y_1_backward(Tensor grad_output, Tensor z) -> Tensor");                                    \
  (m).def("spherical_bessel_y_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");    \
  /* torchscience.cpp:952-954 */                                                                                       \
  (m).def("spherical_bessel_i_0(Tensor z) -> Tensor");                                                                 \
  (m).def("spherical_bessel_i_0_backward(Tensor grad_output, Tensor z) -> Tensor");                                    \
  (m).def("spherical_bessel_i_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");    \
  /* torchscience.cpp:957-959 */                                                                                       \
  (m).def("spherical_bessel_i_1(Tensor z) -> Tensor");                                                                 \
  (m).def("spherical_bessel_i_1_backward(Tensor grad_output, Tensor z) -> Tensor");                                    \
  (m).def("spherical_bessel_i_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");    \
  /* torchscience.cpp:967-969 */                                                                                       \
  (m).def("spherical_bessel_k_0(Tensor z) -> Tensor");                                                                 \
  (m).def("spherical_bessel_k_0_backward(Tensor grad_output, Tensor z) -> Tensor");                                    \
  (m).def("spherical_bessel_k_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");    \
  /* torchscience.cpp:972-974 */                                                                                       \
  (m).def("spherical_bessel_k_1(Tensor z) -> Tensor");                                                                 \
  (m).def("spherical_bessel_k_1_backward(Tensor grad_output, Tensor z) -> Tensor");                                    \
  (m).def("spherical_bessel_k_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");    \
  /* torchscience.cpp:932-934 */                                                                                       \
  (m).def("spherical_bessel_j(Tensor n, Tensor z) -> Tensor");                                                         \
  (m).def("spherical_bessel_j_backward(Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor)");                  \
  (m).def(                                                                                                             \
      "spherical_bessel_j_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> "     \
      "(Tensor, Tensor, Tensor)");                                                                                     \
  /* torchscience.cpp:947-949 */                                                                                       \
  (m).def("spherical_bessel_y(Tensor n, Tensor z) -> Tensor");                                                         \
  (m).def("spherical_bessel_y_backward(Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor)");                  \
  (m).def(                                                                                                             \
      "spherical_bessel_y_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> "     \
      "(Tensor, Tensor, Tensor)");                                                                                     \
  /* torchscience.cpp:962-964 */                                                                                       \
  (m).def("spherical_bessel_i(Tensor n, Tensor z) -> Tensor");                                                         \
  (m).def("spherical_bessel_i_backward(Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor)");                  \
  (m).def(                                                                                                             \
      "spherical_bessel_i_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> "     \
      "(Tensor, Tensor, Tensor)");                                                                                     \
  /* torchscience.cpp:977-979 */                                                                                       \
  (m).def("spherical_bessel_k(Tensor n, Tensor z) -> Tensor");                                                         \
  (m).def("spherical_bessel_k_backward(Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor)");                  \
  (m).def(                                                                                                             \
      "spherical_bessel_k_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> "     \
      "(Tensor, Tensor, Tensor)");                                                                                     \
  /* torchscience.cpp:833-835 */                                                                                     \
  (m).def("incomplete_beta(Tensor x, Tensor a, Tensor b) -> Tensor");                                                \
  (m).def(                                                                                                           \
      "incomplete_beta_backward(Tensor grad_output, Tensor x, Tensor a, Tensor b) -> (Tensor, Tensor, Tensor)");     \
  (m).def(                                                                                                           \
      "incomplete_beta_backward_backward(Tensor gg_x, Tensor gg_a, Tensor gg_b, Tensor grad_output, Tensor x, "      \
      "Tensor a, Tensor b) -> (Tensor, Tensor, Tensor, Tensor)");                                                    \
  /* torchscience.cpp:837-839 */                                                                                     \
  (m).def("hypergeometric_2_f_1(Tensor a, Tensor b, Tensor c, Tensor z) -> Tensor");                                 \
  (m).def(                                                                                                           \
      "hypergeometric_2_f_1_backward(Tensor grad_output, Tensor a, Tensor b, Tensor c, Tensor z) -> (Tensor, Tensor, " \
      "Tensor, Tensor)");                                                                                            \
  (m).def(                                                                                                           \
      "hypergeometric_2_f_1_backward_backward(Tensor gg_a, Tensor gg_b, Tensor gg_c, Tensor gg_z, Tensor "           \
      "grad_output, Tensor a, Tensor b, Tensor c, Tensor z) -> (Tensor, Tensor, Tensor, Tensor, Tensor)");           \
  /* torchscience.cpp:849-851 */                                                                                     \
  (m).def("log_gamma(Tensor z) -> Tensor");                                                                          \
  (m).def("log_gamma_backward(Tensor grad_output, Tensor z) -> Tensor");                                             \
  (m).def("log_gamma_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");             \
  /* torchscience.cpp:853-855 */                                                                                     \
  (m).def("regularized_gamma_p(Tensor a, Tensor x) -> Tensor");                                                      \
  (m).def("regularized_gamma_p_backward(Tensor grad, Tensor a, Tensor x) -> (Tensor, Tensor)");                      \
  (m).def(                                                                                                           \
      "regularized_gamma_p_backward_backward(Tensor grad_grad_a, Tensor grad_grad_x, Tensor grad, Tensor a, Tensor " \
      "x) -> (Tensor, Tensor, Tensor)");                                                                             \
  /* torchscience.cpp:857-859 */                                                                                     \
  (m).def("regularized_gamma_q(Tensor a, Tensor x) -> Tensor");                                                      \
  (m).def("regularized_gamma_q_backward(Tensor grad, Tensor a, Tensor x) -> (Tensor, Tensor)");                      \
  (m).def(                                                                                                           \
      "regularized_gamma_q_backward_backward(Tensor grad_grad_a, Tensor grad_grad_x, Tensor grad, Tensor a, Tensor " \
      "x) -> (Tensor, Tensor, Tensor)");                                                                             \
  /* torchscience.cpp:872-874 */                                                                                     \
  (m).def("bessel_j_0(Tensor z) -> Tensor");                                                                         \
  (m).def("bessel_j_0_backward(Tensor grad_output, Tensor z) -> Tensor");                                            \
  (m).def("bessel_j_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)");            \
  /* torchscience.cpp:902-904 */                                                                                     \
  (m).def("bessel_j(Tensor n, Tensor z) -> Tensor");                                                                 \
  (m).def("bessel_j_backward(Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor)");                          \
  (m).def(                                                                                                           \
      "bessel_j_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> (Tensor, "    \
      "Tensor, Tensor)");                                                                                            \
  /* torchscience.cpp:907-909 */                                                                                     \
  (m).def("bessel_y(Tensor n, Tensor z) -> Tensor");                                                                 \
  (m).def("bessel_y_backward(Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor)");                          \
  (m).def(                                                                                                           \
      "bessel_y_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> (Tensor, "    \
      "Tensor, Tensor)");                                                                                            \
  /* torchscience.cpp:912-914 */                                                                                     \
  (m).def("modified_bessel_k(Tensor n, Tensor z) -> Tensor");                                                        \
  (m).def("modified_bessel_k_backward(Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor)");                 \
  (m).def(                                                                                                           \
      "modified_bessel_k_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> "    \
      "(Tensor, Tensor, Tensor)");                                                                                   \
  /* torchscience.cpp:917-919 */                                                                                     \
  (m).def("modified_bessel_i(Tensor n, Tensor z) -> Tensor");                                                        \
  (m).def("modified_bessel_i_backward(Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor)");                 \
  (m).def(                                                                                                           \
      "modified_bessel_i_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> "    \
      "(Tensor, Tensor, Tensor)");                                                                                   \
  /* torchscience.cpp:1015-1017 */                                                                                   \
  (m).def("complete_legendre_elliptic_integral_k(Tensor m) -> Tensor");                                              \
  (m).def("complete_legendre_elliptic_integral_k_backward(Tensor grad_output, Tensor m) -> Tensor");                 \
  (m).def(                                                                                                           \
      "complete_legendre_elliptic_integral_k_backward_backward(Tensor gg_m, Tensor grad_output, Tensor m) -> "       \
      "(Tensor, Tensor)");                                                                                           \
  /* torchscience.cpp:1019-1021 */                                                                                   \
  (m).def("complete_legendre_elliptic_integral_e(Tensor m) -> Tensor");                                              \
  (m).def("complete_legendre_elliptic_integral_e_backward(Tensor grad_output, Tensor m) -> Tensor");                 \
  (m).def(                                                                                                           \
      "complete_legendre_elliptic_integral_e_backward_backward(Tensor gg_m, Tensor grad_output, Tensor m) -> "       \
      "(Tensor, Tensor)");

// Schemas of the probability callers of the incomplete gamma (torchscience.cpp:1881-1888, 1909-1912,
// 1923-1924), registered by this package only.
#define TSB_DEFINE_PROBABILITY_SCHEMAS(m)                                                                             \
  (m).def("chi2_cumulative_distribution(Tensor x, Tensor df) -> Tensor");                                            \
  (m).def("chi2_cumulative_distribution_backward(Tensor grad, Tensor x, Tensor df) -> (Tensor, Tensor)");            \
  (m).def("gamma_cumulative_distribution(Tensor x, Tensor shape, Tensor scale) -> Tensor");                          \
  (m).def(                                                                                                           \
      "gamma_cumulative_distribution_backward(Tensor grad, Tensor x, Tensor shape, Tensor scale) -> (Tensor, Tensor, " \
      "Tensor)");                                                                                                    \
  (m).def("poisson_cumulative_distribution(Tensor k, Tensor rate) -> Tensor");                                       \
  (m).def("poisson_cumulative_distribution_backward(Tensor grad, Tensor k, Tensor rate) -> (Tensor, Tensor)");       \
  (m).def("chi2_survival(Tensor x, Tensor df) -> Tensor");                                                           \
  (m).def("chi2_survival_backward(Tensor grad, Tensor x, Tensor df) -> (Tensor, Tensor)");                           \
  (m).def("chi2_probability_density(Tensor x, Tensor df) -> Tensor");                                               \
  (m).def("chi2_probability_density_backward(Tensor grad, Tensor x, Tensor df) -> (Tensor, Tensor)");               \
  (m).def("gamma_probability_density(Tensor x, Tensor shape, Tensor scale) -> Tensor");                             \
  (m).def(                                                                                                           \
      "gamma_probability_density_backward(Tensor grad, Tensor x, Tensor shape, Tensor scale) -> (Tensor, Tensor, "   \
      "Tensor)");
