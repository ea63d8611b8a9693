// Thin C ABI over the reference's own scalar kernels, for tests and the CPU
// baseline.  This file is oracle infrastructure: it is compiled (by
// oracle/build_ref.py) against the reference's headers where they lie
// (src/torchscience/csrc/kernel/special_functions/*.h) into
// oracle/_ref/libref_scalar.so, and is never part of the product.
//
// ref_eval(name, pass, dtype, in, out, n) runs the reference template
// `name` (pass 0), `name_backward` (pass 1) or `name_backward_backward`
// (pass 2) elementwise over n contiguous elements, OpenMP-parallel.
// dtype 0 = float, 1 = double.  Returns 0, or -1 for an unknown name/pass.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <cstring>
#include <tuple>

#include "kernel/probability/chi2_cumulative_distribution.h"
#include "kernel/probability/chi2_cumulative_distribution_backward.h"
#include "kernel/probability/gamma_cumulative_distribution.h"
#include "kernel/probability/gamma_cumulative_distribution_backward.h"
#include "kernel/probability/poisson_cumulative_distribution.h"
#include "kernel/probability/poisson_cumulative_distribution_backward.h"
#include "kernel/probability/chi2_survival.h"
#include "kernel/probability/chi2_survival_backward.h"
#include "kernel/probability/gamma_probability_density.h"
#include "kernel/probability/gamma_probability_density_backward.h"
#include "kernel/probability/chi2_probability_density.h"
#include "kernel/probability/chi2_probability_density_backward.h"
#include "kernel/special_functions/beta.h"
#include "kernel/special_functions/beta_backward.h"
#include "kernel/special_functions/beta_backward_backward.h"
#include "kernel/special_functions/incomplete_beta.h"
#include "kernel/special_functions/incomplete_beta_backward.h"
#include "kernel/special_functions/incomplete_beta_backward_backward.h"
#include "kernel/special_functions/log_beta.h"
#include "kernel/special_functions/log_beta_backward.h"
#include "kernel/special_functions/log_beta_backward_backward.h"
#include "kernel/special_functions/polygamma.h"
#include "kernel/special_functions/polygamma_backward.h"
#include "kernel/special_functions/polygamma_backward_backward.h"
#include "kernel/special_functions/bessel_j_1.h"
#include "kernel/special_functions/bessel_j_1_backward.h"
#include "kernel/special_functions/bessel_j_1_backward_backward.h"
#include "kernel/special_functions/bessel_y_0.h"
#include "kernel/special_functions/bessel_y_0_backward.h"
#include "kernel/special_functions/bessel_y_0_backward_backward.h"
#include "kernel/special_functions/bessel_y_1.h"
#include "kernel/special_functions/bessel_y_1_backward.h"
#include "kernel/special_functions/bessel_y_1_backward_backward.h"
#include "kernel/special_functions/modified_bessel_i_0.h"
#include "kernel/special_functions/modified_bessel_i_0_backward.h"
#include "kernel/special_functions/modified_bessel_i_0_backward_backward.h"
#include "kernel/special_functions/modified_bessel_i_1.h"
#include "kernel/special_functions/modified_bessel_i_1_backward.h"
#include "kernel/special_functions/modified_bessel_i_1_backward_backward.h"
#include "kernel/special_functions/modified_bessel_k_0.h"
#include "kernel/special_functions/modified_bessel_k_0_backward.h"
#include "kernel/special_functions/modified_bessel_k_0_backward_backward.h"
#include "kernel/special_functions/modified_bessel_k_1.h"
#include "kernel/special_functions/modified_bessel_k_1_backward.h"
#include "kernel/special_functions/modified_bessel_k_1_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_j_0.h"
#include "kernel/special_functions/spherical_bessel_j_0_backward.h"
#include "kernel/special_functions/spherical_bessel_j_0_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_j_1.h"
#include "kernel/special_functions/spherical_bessel_j_1_backward.h"
#include "kernel/special_functions/spherical_bessel_j_1_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_y_0.h"
#include "kernel/special_functions/spherical_bessel_y_0_backward.h"
#include "kernel/special_functions/spherical_bessel_y_0_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_y_1.h"
#include "kernel/special_functions/spherical_bessel_y_1_backward.h"
#include "kernel/special_functions/spherical_bessel_y_1_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_i_0.h"
#include "kernel/special_functions/spherical_bessel_i_0_backward.h"
#include "kernel/special_functions/spherical_bessel_i_0_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_i_1.h"
#include "kernel/special_functions/spherical_bessel_i_1_backward.h"
#include "kernel/special_functions/spherical_bessel_i_1_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_k_0.h"
#include "kernel/special_functions/spherical_bessel_k_0_backward.h"
#include "kernel/special_functions/spherical_bessel_k_0_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_k_1.h"
#include "kernel/special_functions/spherical_bessel_k_1_backward.h"
#include "kernel/special_functions/spherical_bessel_k_1_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_j.h"
#include "kernel/special_functions/spherical_bessel_j_backward.h"
#include "kernel/special_functions/spherical_bessel_j_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_y.h"
#include "kernel/special_functions/spherical_bessel_y_backward.h"
#include "kernel/special_functions/spherical_bessel_y_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_i.h"
#include "kernel/special_functions/spherical_bessel_i_backward.h"
#include "kernel/special_functions/spherical_bessel_i_backward_backward.h"
#include "kernel/special_functions/spherical_bessel_k.h"
#include "kernel/special_functions/spherical_bessel_k_backward.h"
#include "kernel/special_functions/spherical_bessel_k_backward_backward.h"
#include "kernel/special_functions/bessel_j.h"
#include "kernel/special_functions/bessel_j_0.h"
#include "kernel/special_functions/bessel_j_0_backward.h"
#include "kernel/special_functions/bessel_j_0_backward_backward.h"
#include "kernel/special_functions/bessel_j_backward.h"
#include "kernel/special_functions/bessel_j_backward_backward.h"
#include "kernel/special_functions/bessel_y.h"
#include "kernel/special_functions/bessel_y_backward.h"
#include "kernel/special_functions/bessel_y_backward_backward.h"
#include "kernel/special_functions/complete_legendre_elliptic_integral_e.h"
#include "kernel/special_functions/complete_legendre_elliptic_integral_e_backward.h"
#include "kernel/special_functions/complete_legendre_elliptic_integral_e_backward_backward.h"
#include "kernel/special_functions/complete_legendre_elliptic_integral_k.h"
#include "kernel/special_functions/complete_legendre_elliptic_integral_k_backward.h"
#include "kernel/special_functions/complete_legendre_elliptic_integral_k_backward_backward.h"
#include "kernel/special_functions/digamma.h"
#include "kernel/special_functions/digamma_backward.h"
#include "kernel/special_functions/digamma_backward_backward.h"
#include "kernel/special_functions/gamma.h"
#include "kernel/special_functions/gamma_backward.h"
#include "kernel/special_functions/gamma_backward_backward.h"
#include "kernel/special_functions/hypergeometric_2_f_1.h"
#include "kernel/special_functions/hypergeometric_2_f_1_backward.h"
#include "kernel/special_functions/hypergeometric_2_f_1_backward_backward.h"
#include "kernel/special_functions/log_gamma.h"
#include "kernel/special_functions/log_gamma_backward.h"
#include "kernel/special_functions/log_gamma_backward_backward.h"
#include "kernel/special_functions/modified_bessel_i.h"
#include "kernel/special_functions/modified_bessel_i_backward.h"
#include "kernel/special_functions/modified_bessel_i_backward_backward.h"
#include "kernel/special_functions/modified_bessel_k.h"
#include "kernel/special_functions/modified_bessel_k_backward.h"
#include "kernel/special_functions/modified_bessel_k_backward_backward.h"
#include "kernel/special_functions/regularized_gamma_p.h"
#include "kernel/special_functions/regularized_gamma_p_backward.h"
#include "kernel/special_functions/regularized_gamma_p_backward_backward.h"
#include "kernel/special_functions/regularized_gamma_q.h"
#include "kernel/special_functions/regularized_gamma_q_backward.h"
#include "kernel/special_functions/regularized_gamma_q_backward_backward.h"
#include "kernel/special_functions/trigamma.h"
#include "kernel/special_functions/trigamma_backward.h"
#include "kernel/special_functions/trigamma_backward_backward.h"

namespace sf = torchscience::kernel::special_functions;
namespace pr = torchscience::kernel::probability;

namespace {

template <typename T>
void put(void* const* out, int64_t i, int k, T v) {
  static_cast<T*>(out[k])[i] = v;
}
template <typename T, typename A, typename B>
void put(void* const* out, int64_t i, std::tuple<A, B> v) {
  put<T>(out, i, 0, std::get<0>(v));
  put<T>(out, i, 1, std::get<1>(v));
}
template <typename T, typename A, typename B, typename C>
void put(void* const* out, int64_t i, std::tuple<A, B, C> v) {
  put<T>(out, i, 0, std::get<0>(v));
  put<T>(out, i, 1, std::get<1>(v));
  put<T>(out, i, 2, std::get<2>(v));
}
template <typename T, typename A, typename B, typename C, typename D>
void put(void* const* out, int64_t i, std::tuple<A, B, C, D> v) {
  put<T>(out, i, 0, std::get<0>(v));
  put<T>(out, i, 1, std::get<1>(v));
  put<T>(out, i, 2, std::get<2>(v));
  put<T>(out, i, 3, std::get<3>(v));
}
template <typename T, typename A, typename B, typename C, typename D, typename E>
void put(void* const* out, int64_t i, std::tuple<A, B, C, D, E> v) {
  put<T>(out, i, 0, std::get<0>(v));
  put<T>(out, i, 1, std::get<1>(v));
  put<T>(out, i, 2, std::get<2>(v));
  put<T>(out, i, 3, std::get<3>(v));
  put<T>(out, i, 4, std::get<4>(v));
}
template <typename T>
void put(void* const* out, int64_t i, T v) {
  put<T>(out, i, 0, v);
}

template <typename T>
T arg_at(const void* const* in, int k, int64_t i) {
  return static_cast<const T*>(in[k])[i];
}

}  // namespace

#define ARG(k) arg_at<T>(in, k, i)
#define LOOP(expr)                                         \
  do {                                                     \
    _Pragma("omp parallel for schedule(dynamic, 256)")     \
    for (int64_t i = 0; i < n; ++i) put<T>(out, i, expr); \
    return 0;                                              \
  } while (0)

#define UNARY(nm)                                                                          \
  if (std::strcmp(name, #nm) == 0) {                                                       \
    if (pass == 0) LOOP(sf::nm(ARG(0)));                                                   \
    if (pass == 1) LOOP(sf::nm##_backward(ARG(0), ARG(1)));                                \
    if (pass == 2) LOOP(sf::nm##_backward_backward(ARG(0), ARG(1), ARG(2)));               \
    return -1;                                                                             \
  }
#define BINARY(nm)                                                                         \
  if (std::strcmp(name, #nm) == 0) {                                                       \
    if (pass == 0) LOOP(sf::nm(ARG(0), ARG(1)));                                           \
    if (pass == 1) LOOP(sf::nm##_backward(ARG(0), ARG(1), ARG(2)));                        \
    if (pass == 2) LOOP(sf::nm##_backward_backward(ARG(0), ARG(1), ARG(2), ARG(3), ARG(4))); \
    return -1;                                                                             \
  }

template <typename T>
static int eval_typed(const char* name, int pass, const void* const* in, void* const* out, int64_t n) {
  UNARY(log_gamma)
  UNARY(gamma)
  UNARY(digamma)
  UNARY(trigamma)
  UNARY(bessel_j_0)
  UNARY(spherical_bessel_j_0)
  UNARY(spherical_bessel_j_1)
  UNARY(spherical_bessel_y_0)
  UNARY(spherical_bessel_y_1)
  UNARY(spherical_bessel_i_0)
  UNARY(spherical_bessel_i_1)
  UNARY(spherical_bessel_k_0)
  UNARY(spherical_bessel_k_1)
  UNARY(bessel_j_1)
  UNARY(bessel_y_0)
  UNARY(bessel_y_1)
  UNARY(modified_bessel_i_0)
  UNARY(modified_bessel_i_1)
  UNARY(modified_bessel_k_0)
  UNARY(modified_bessel_k_1)
  UNARY(complete_legendre_elliptic_integral_k)
  UNARY(complete_legendre_elliptic_integral_e)
  BINARY(regularized_gamma_p)
  BINARY(regularized_gamma_q)
  BINARY(bessel_j)
  BINARY(bessel_y)
  BINARY(modified_bessel_i)
  BINARY(modified_bessel_k)
  BINARY(spherical_bessel_j)
  BINARY(spherical_bessel_y)
  BINARY(spherical_bessel_i)
  BINARY(spherical_bessel_k)
  BINARY(log_beta)
  BINARY(beta)
  BINARY(polygamma)
  if (std::strcmp(name, "gamma_cumulative_distribution") == 0) {
    if (pass == 0) LOOP(pr::gamma_cumulative_distribution(ARG(0), ARG(1), ARG(2)));
    if (pass == 1) LOOP(pr::gamma_cumulative_distribution_backward(ARG(0), ARG(1), ARG(2), ARG(3)));
    return -1;
  }
  if (std::strcmp(name, "chi2_cumulative_distribution") == 0) {
    if (pass == 0) LOOP(pr::chi2_cumulative_distribution(ARG(0), ARG(1)));
    if (pass == 1) LOOP(pr::chi2_cumulative_distribution_backward(ARG(0), ARG(1), ARG(2)));
    return -1;
  }
  if (std::strcmp(name, "poisson_cumulative_distribution") == 0) {
    if (pass == 0) LOOP(pr::poisson_cumulative_distribution(ARG(0), ARG(1)));
    if (pass == 1) LOOP(pr::poisson_cumulative_distribution_backward(ARG(0), ARG(1), ARG(2)));
    return -1;
  }
  if (std::strcmp(name, "chi2_survival") == 0) {
    if (pass == 0) LOOP(pr::chi2_survival(ARG(0), ARG(1)));
    if (pass == 1) LOOP(pr::chi2_survival_backward(ARG(0), ARG(1), ARG(2)));
    return -1;
  }
  if (std::strcmp(name, "gamma_probability_density") == 0) {
    if (pass == 0) LOOP(pr::gamma_probability_density(ARG(0), ARG(1), ARG(2)));
    if (pass == 1) LOOP(pr::gamma_probability_density_backward(ARG(0), ARG(1), ARG(2), ARG(3)));
    return -1;
  }
  if (std::strcmp(name, "chi2_probability_density") == 0) {
    if (pass == 0) LOOP(pr::chi2_probability_density(ARG(0), ARG(1)));
    if (pass == 1) LOOP(pr::chi2_probability_density_backward(ARG(0), ARG(1), ARG(2)));
    return -1;
  }
  if (std::strcmp(name, "incomplete_beta") == 0) {
    if (pass == 0) LOOP(sf::incomplete_beta(ARG(0), ARG(1), ARG(2)));
    if (pass == 1) LOOP(sf::incomplete_beta_backward(ARG(0), ARG(1), ARG(2), ARG(3)));
    if (pass == 2) LOOP(sf::incomplete_beta_backward_backward(ARG(0), ARG(1), ARG(2), ARG(3), ARG(4), ARG(5), ARG(6)));
    return -1;
  }
  if (std::strcmp(name, "hypergeometric_2_f_1") == 0) {
    if (pass == 0) LOOP(sf::hypergeometric_2_f_1(ARG(0), ARG(1), ARG(2), ARG(3)));
    if (pass == 1) LOOP(sf::hypergeometric_2_f_1_backward(ARG(0), ARG(1), ARG(2), ARG(3), ARG(4)));
    if (pass == 2)
      LOOP(sf::hypergeometric_2_f_1_backward_backward(ARG(0), ARG(1), ARG(2), ARG(3), ARG(4), ARG(5), ARG(6), ARG(7),
                                                      ARG(8)));
    return -1;
  }
  return -1;
}

extern "C" int ref_eval(const char* name, int pass, int dtype, const void* const* in, void* const* out, int64_t n) {
  if (dtype == 1) return eval_typed<double>(name, pass, in, out, n);
  if (dtype == 0) return eval_typed<float>(name, pass, in, out, n);
  return -1;
}
