// Oracle infrastructure, never part of the product: builds the reference's
// own CPU operators for the accelerated special functions (TensorIterator +
// at::native::cpu_kernel over the scalar templates, with the reference's
// Meta, Autograd and Autocast wrappers) as a standalone torch op library,
// oracle/_ref/libtorchscience_ref.so.  It is compiled by oracle/build_ref.py
// against the reference's headers where they lie (src/torchscience/csrc/**);
// the macro invocations below mirror cpu/special_functions.h,
// meta/special_functions.h, autograd/special_functions.h and
// autocast/special_functions.h for the ops on the path.  `bench.py --impl
// reference` loads it (in a process that does not load torchscience_b200) to
// time the reference's CPU path.
#include <algorithm>
#include <cmath>
#include <limits>

#include "autocast/macros.h"
#include "autograd/macros.h"
#include "cpu/macros.h"
#include "meta/macros.h"
#include "schemas.h"

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

TORCH_LIBRARY(torchscience, m) { TSB_DEFINE_TORCHSCIENCE_SCHEMAS(m) }

// CPU (cpu/special_functions.h:9,15,21,45,63,69,75,93,129,135,141,147,200,206)
TORCHSCIENCE_CPU_POINTWISE_UNARY_OPERATOR_WITH_COMPLEX(gamma, z)
TORCHSCIENCE_CPU_POINTWISE_UNARY_OPERATOR_WITH_COMPLEX(digamma, z)
TORCHSCIENCE_CPU_POINTWISE_UNARY_OPERATOR_WITH_COMPLEX(trigamma, z)
TORCHSCIENCE_CPU_POINTWISE_QUATERNARY_OPERATOR_WITH_COMPLEX(hypergeometric_2_f_1, a, b, c, z)
TORCHSCIENCE_CPU_POINTWISE_UNARY_OPERATOR_WITH_COMPLEX(log_gamma, z)
TORCHSCIENCE_CPU_POINTWISE_BINARY_OPERATOR(regularized_gamma_p, a, x)
TORCHSCIENCE_CPU_POINTWISE_BINARY_OPERATOR(regularized_gamma_q, a, x)
TORCHSCIENCE_CPU_POINTWISE_UNARY_OPERATOR_WITH_COMPLEX(bessel_j_0, z)
TORCHSCIENCE_CPU_POINTWISE_BINARY_OPERATOR_WITH_COMPLEX(bessel_j, n, z)
TORCHSCIENCE_CPU_POINTWISE_BINARY_OPERATOR_WITH_COMPLEX(bessel_y, n, z)
TORCHSCIENCE_CPU_POINTWISE_BINARY_OPERATOR_WITH_COMPLEX(modified_bessel_k, n, z)
TORCHSCIENCE_CPU_POINTWISE_BINARY_OPERATOR_WITH_COMPLEX(modified_bessel_i, n, z)
TORCHSCIENCE_CPU_POINTWISE_UNARY_OPERATOR_WITH_COMPLEX(complete_legendre_elliptic_integral_k, m)
TORCHSCIENCE_CPU_POINTWISE_UNARY_OPERATOR_WITH_COMPLEX(complete_legendre_elliptic_integral_e, m)

// Meta (meta/special_functions.h)
TORCHSCIENCE_META_POINTWISE_UNARY_OPERATOR(gamma, z)
TORCHSCIENCE_META_POINTWISE_UNARY_OPERATOR(digamma, z)
TORCHSCIENCE_META_POINTWISE_UNARY_OPERATOR(trigamma, z)
TORCHSCIENCE_META_POINTWISE_QUATERNARY_OPERATOR(hypergeometric_2_f_1, a, b, c, z)
TORCHSCIENCE_META_POINTWISE_UNARY_OPERATOR(log_gamma, z)
TORCHSCIENCE_META_POINTWISE_BINARY_OPERATOR(regularized_gamma_p, a, x)
TORCHSCIENCE_META_POINTWISE_BINARY_OPERATOR(regularized_gamma_q, a, x)
TORCHSCIENCE_META_POINTWISE_UNARY_OPERATOR(bessel_j_0, z)
TORCHSCIENCE_META_POINTWISE_BINARY_OPERATOR(bessel_j, n, z)
TORCHSCIENCE_META_POINTWISE_BINARY_OPERATOR(bessel_y, n, z)
TORCHSCIENCE_META_POINTWISE_BINARY_OPERATOR(modified_bessel_k, n, z)
TORCHSCIENCE_META_POINTWISE_BINARY_OPERATOR(modified_bessel_i, n, z)
TORCHSCIENCE_META_POINTWISE_UNARY_OPERATOR(complete_legendre_elliptic_integral_k, m)
TORCHSCIENCE_META_POINTWISE_UNARY_OPERATOR(complete_legendre_elliptic_integral_e, m)

// Autograd (autograd/special_functions.h:5-38)
TORCHSCIENCE_AUTOGRAD_POINTWISE_UNARY_OPERATOR(gamma, Gamma, z)
TORCHSCIENCE_AUTOGRAD_POINTWISE_UNARY_OPERATOR(digamma, Digamma, z)
TORCHSCIENCE_AUTOGRAD_POINTWISE_UNARY_OPERATOR(trigamma, Trigamma, z)
TORCHSCIENCE_AUTOGRAD_POINTWISE_QUATERNARY_OPERATOR(hypergeometric_2_f_1, Hypergeometric2F1, a, b, c, z)
TORCHSCIENCE_AUTOGRAD_POINTWISE_UNARY_OPERATOR(log_gamma, LogGamma, z)
TORCHSCIENCE_AUTOGRAD_POINTWISE_BINARY_OPERATOR(regularized_gamma_p, RegularizedGammaP, a, x)
TORCHSCIENCE_AUTOGRAD_POINTWISE_BINARY_OPERATOR(regularized_gamma_q, RegularizedGammaQ, a, x)
TORCHSCIENCE_AUTOGRAD_POINTWISE_UNARY_OPERATOR(bessel_j_0, BesselJ0, z)
TORCHSCIENCE_AUTOGRAD_POINTWISE_BINARY_OPERATOR(bessel_j, BesselJ, n, z)
TORCHSCIENCE_AUTOGRAD_POINTWISE_BINARY_OPERATOR(bessel_y, BesselY, n, z)
TORCHSCIENCE_AUTOGRAD_POINTWISE_BINARY_OPERATOR(modified_bessel_k, ModifiedBesselK, n, z)
TORCHSCIENCE_AUTOGRAD_POINTWISE_BINARY_OPERATOR(modified_bessel_i, ModifiedBesselI, n, z)
TORCHSCIENCE_AUTOGRAD_POINTWISE_UNARY_OPERATOR(complete_legendre_elliptic_integral_k, CompleteLegendreEllipticIntegralK, m)
TORCHSCIENCE_AUTOGRAD_POINTWISE_UNARY_OPERATOR(complete_legendre_elliptic_integral_e, CompleteLegendreEllipticIntegralE, m)
