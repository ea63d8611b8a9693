"""Special functions with the reference's Python API (torchscience.special_functions).

Each function is a thin call into ``torch.ops.torchscience.<name>``, registered by
this package's native library for CUDA tensors: broadcasting and dtype promotion
follow TensorIterator, float16/bfloat16/float32 inputs use the mixed-precision
kernels and float64 inputs the FP64 kernels; integer and complex inputs raise
NotImplementedError and CPU tensors raise RuntimeError.
"""

from __future__ import annotations

import torch
from torch import Tensor

def log_gamma(z: Tensor) -> Tensor:
    """Natural log of |Γ(z)|; +inf at the non-positive integers.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_log_gamma.py:5,115).
    """
    return torch.ops.torchscience.log_gamma(z)


def gamma(z: Tensor) -> Tensor:
    """Gamma function Γ(z); +inf at the non-positive integers.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_gamma.py).
    """
    return torch.ops.torchscience.gamma(z)


def digamma(z: Tensor) -> Tensor:
    """Digamma ψ(z) = d lnΓ(z)/dz; -inf at the non-positive integers.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_digamma.py).
    """
    return torch.ops.torchscience.digamma(z)


def trigamma(z: Tensor) -> Tensor:
    """Trigamma ψ'(z); +inf at the non-positive integers.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_trigamma.py).
    """
    return torch.ops.torchscience.trigamma(z)


def regularized_gamma_p(a: Tensor, x: Tensor) -> Tensor:
    """Regularized lower incomplete gamma P(a, x) = γ(a, x)/Γ(a); NaN for x < 0 or a <= 0.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_regularized_gamma_p.py:9,60).
    """
    return torch.ops.torchscience.regularized_gamma_p(a, x)


def regularized_gamma_q(a: Tensor, x: Tensor) -> Tensor:
    """Regularized upper incomplete gamma Q(a, x) = 1 - P(a, x); NaN for x < 0 or a <= 0.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_regularized_gamma_q.py).
    """
    return torch.ops.torchscience.regularized_gamma_q(a, x)


def complete_legendre_elliptic_integral_k(m: Tensor) -> Tensor:
    """Complete elliptic integral of the first kind K(m) (parameter m = k²); NaN for m > 1, +inf at m = 1.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_complete_legendre_elliptic_integral_k.py:5,149).
    """
    return torch.ops.torchscience.complete_legendre_elliptic_integral_k(m)


def bessel_j_0(z: Tensor) -> Tensor:
    """Bessel function of the first kind of order zero J_0(z).

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_bessel_j_0.py).
    """
    return torch.ops.torchscience.bessel_j_0(z)


def bessel_j(n: Tensor, z: Tensor) -> Tensor:
    """Bessel function of the first kind J_n(z) of real order n.

    For z < 0 returns (-1)^n J_n(|z|) for integer n and cos(πn) J_n(|z|)
    otherwise (the reference's real-valued convention).  Same signature and
    semantics as the reference wrapper (src/torchscience/special_functions/_bessel_j.py:5,193).
    """
    return torch.ops.torchscience.bessel_j(n, z)


def bessel_y(n: Tensor, z: Tensor) -> Tensor:
    """Bessel function of the second kind Y_n(z) of real order n; NaN for z < 0, -inf at z = 0.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_bessel_y.py).
    """
    return torch.ops.torchscience.bessel_y(n, z)


def modified_bessel_i(n: Tensor, z: Tensor) -> Tensor:
    """Modified Bessel function of the first kind I_n(z) of real order n.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_modified_bessel_i.py).
    """
    return torch.ops.torchscience.modified_bessel_i(n, z)


def modified_bessel_k(n: Tensor, z: Tensor) -> Tensor:
    """Modified Bessel function of the second kind K_n(z) of real order n; NaN for z < 0, +inf at z = 0.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_modified_bessel_k.py).
    """
    return torch.ops.torchscience.modified_bessel_k(n, z)


def complete_legendre_elliptic_integral_e(m: Tensor) -> Tensor:
    """Complete elliptic integral of the second kind E(m) (parameter m = k²); NaN for m > 1, E(1) = 1.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_complete_legendre_elliptic_integral_e.py).
    """
    return torch.ops.torchscience.complete_legendre_elliptic_integral_e(m)


def hypergeometric_2_f_1(a: Tensor, b: Tensor, c: Tensor, z: Tensor) -> Tensor:
    """Gauss hypergeometric function 2F1(a, b; c; z) for real arguments; NaN for z > 1.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_hypergeometric_2_f_1.py),
    including its special values (hypergeometric_2_f_1.h:203-295). Every dtype is evaluated in FP64.
    """
    return torch.ops.torchscience.hypergeometric_2_f_1(a, b, c, z)


def polygamma(n: Tensor, z: Tensor) -> Tensor:
    """Polygamma ψ^(n)(z), the order read as the reference reads it (truncated
    toward zero; NaN for n <= -1).  n >= 4 uses the Hurwitz zeta
    (-1)^(n+1) n! ζ(n+1, z) by Euler–Maclaurin summation.  Same signature and
    semantics as the reference wrapper (src/torchscience/special_functions/_polygamma.py:5).
    """
    return torch.ops.torchscience.polygamma(n, z)


def log_beta(a: Tensor, b: Tensor) -> Tensor:
    """ln|B(a, b)| = lnΓ(a) + lnΓ(b) - lnΓ(a+b), formed without the
    cancellation of those sums for large arguments; +inf where Γ(a) or Γ(b)
    has a pole.  Same signature as the reference wrapper
    (src/torchscience/special_functions/_log_beta.py:5).
    """
    return torch.ops.torchscience.log_beta(a, b)


def beta(a: Tensor, b: Tensor) -> Tensor:
    """Beta function B(a, b) = Γ(a)Γ(b)/Γ(a+b), with its sign for negative
    arguments (the reference returns exp(ln|B|)).  Same signature as the
    reference wrapper (src/torchscience/special_functions/_beta.py:5).
    """
    return torch.ops.torchscience.beta(a, b)


def incomplete_beta(z: Tensor, a: Tensor, b: Tensor) -> Tensor:
    """Regularized incomplete beta function I_z(a, b) for 0 < z < 1 and
    a, b > 0: 0 for z <= 0, 1 for z >= 1, NaN for a <= 0 or b <= 0.
    Differentiable in z, a and b (to second order); the a/b derivatives are
    exact to rounding.  Same signature as the reference wrapper
    (src/torchscience/special_functions/_incomplete_beta.py:5).
    """
    return torch.ops.torchscience.incomplete_beta(z, a, b)


def bessel_j_1(z: Tensor) -> Tensor:
    """Bessel function of the first kind of order one, J_1(z) (odd in z).

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_bessel_j_1.py).
    """
    return torch.ops.torchscience.bessel_j_1(z)


def bessel_y_0(z: Tensor) -> Tensor:
    """Bessel function of the second kind of order zero, Y_0(z); NaN for z < 0, -inf at 0.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_bessel_y_0.py).
    """
    return torch.ops.torchscience.bessel_y_0(z)


def bessel_y_1(z: Tensor) -> Tensor:
    """Bessel function of the second kind of order one, Y_1(z); NaN for z < 0, -inf at 0.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_bessel_y_1.py).
    """
    return torch.ops.torchscience.bessel_y_1(z)


def modified_bessel_i_0(z: Tensor) -> Tensor:
    """Modified Bessel function of the first kind of order zero, I_0(z) (even in z).

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_modified_bessel_i_0.py).
    """
    return torch.ops.torchscience.modified_bessel_i_0(z)


def modified_bessel_i_1(z: Tensor) -> Tensor:
    """Modified Bessel function of the first kind of order one, I_1(z) (odd in z).

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_modified_bessel_i_1.py).
    """
    return torch.ops.torchscience.modified_bessel_i_1(z)


def modified_bessel_k_0(z: Tensor) -> Tensor:
    """Modified Bessel function of the second kind of order zero, K_0(z); NaN for z < 0, +inf at 0.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_modified_bessel_k_0.py).
    """
    return torch.ops.torchscience.modified_bessel_k_0(z)


def modified_bessel_k_1(z: Tensor) -> Tensor:
    """Modified Bessel function of the second kind of order one, K_1(z); NaN for z < 0, +inf at 0.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_modified_bessel_k_1.py).
    """
    return torch.ops.torchscience.modified_bessel_k_1(z)


def spherical_bessel_j_0(z: Tensor) -> Tensor:
    """Spherical Bessel function j_0(z) = sin(z)/z.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_j_0.py).
    """
    return torch.ops.torchscience.spherical_bessel_j_0(z)


def spherical_bessel_j_1(z: Tensor) -> Tensor:
    """Spherical Bessel function j_1(z) = sin(z)/z² - cos(z)/z (series below |z| = 1).

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_j_1.py).
    """
    return torch.ops.torchscience.spherical_bessel_j_1(z)


def spherical_bessel_y_0(z: Tensor) -> Tensor:
    """Spherical Bessel function y_0(z) = -cos(z)/z; -inf at 0.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_y_0.py).
    """
    return torch.ops.torchscience.spherical_bessel_y_0(z)


def spherical_bessel_y_1(z: Tensor) -> Tensor:
    """Spherical Bessel function y_1(z) = -cos(z)/z² - sin(z)/z; -inf at 0.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_y_1.py).
    """
    return torch.ops.torchscience.spherical_bessel_y_1(z)


def spherical_bessel_i_0(z: Tensor) -> Tensor:
    """Modified spherical Bessel function i_0(z) = sinh(z)/z.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_i_0.py).
    """
    return torch.ops.torchscience.spherical_bessel_i_0(z)


def spherical_bessel_i_1(z: Tensor) -> Tensor:
    """Modified spherical Bessel function i_1(z) = cosh(z)/z - sinh(z)/z² (series below |z| = 1).

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_i_1.py).
    """
    return torch.ops.torchscience.spherical_bessel_i_1(z)


def spherical_bessel_k_0(z: Tensor) -> Tensor:
    """Modified spherical Bessel function k_0(z) = (π/2) e^-z / z.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_k_0.py).
    """
    return torch.ops.torchscience.spherical_bessel_k_0(z)


def spherical_bessel_k_1(z: Tensor) -> Tensor:
    """Modified spherical Bessel function k_1(z) = (π/2)(1 + z) e^-z / z²; +inf below |z| = 1e-12.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_k_1.py).
    """
    return torch.ops.torchscience.spherical_bessel_k_1(z)


def spherical_bessel_j(n: Tensor, z: Tensor) -> Tensor:
    """Spherical Bessel function of the first kind j_n(z) = sqrt(π/(2z)) J_{n+1/2}(z) of real order n.

    For z < 0 the reference's real-valued conventions apply ((-1)^n or cos(πn) factors).  Same
    signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_j.py).
    """
    return torch.ops.torchscience.spherical_bessel_j(n, z)


def spherical_bessel_y(n: Tensor, z: Tensor) -> Tensor:
    """Spherical Bessel function of the second kind y_n(z) = sqrt(π/(2z)) Y_{n+1/2}(z) of real order n.

    For z < 0 the reference's real-valued conventions apply ((-1)^n or cos(πn) factors).  Same
    signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_y.py).
    """
    return torch.ops.torchscience.spherical_bessel_y(n, z)


def spherical_bessel_i(n: Tensor, z: Tensor) -> Tensor:
    """Modified spherical Bessel function i_n(z) = sqrt(π/(2z)) I_{n+1/2}(z) of real order n.

    For z < 0 the reference's real-valued conventions apply ((-1)^n or cos(πn) factors).  Same
    signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_i.py).
    """
    return torch.ops.torchscience.spherical_bessel_i(n, z)


def spherical_bessel_k(n: Tensor, z: Tensor) -> Tensor:
    """Modified spherical Bessel function k_n(z) = sqrt(π/(2z)) K_{n+1/2}(z) of real order n; NaN for z < 0.

    For z < 0 the reference's real-valued conventions apply ((-1)^n or cos(πn) factors).  Same
    signature and semantics as the reference wrapper (src/torchscience/special_functions/_spherical_bessel_k.py).
    """
    return torch.ops.torchscience.spherical_bessel_k(n, z)


__all__ = [
    "bessel_j",
    "bessel_j_0",
    "bessel_j_1",
    "bessel_y",
    "bessel_y_0",
    "bessel_y_1",
    "beta",
    "complete_legendre_elliptic_integral_e",
    "complete_legendre_elliptic_integral_k",
    "digamma",
    "gamma",
    "hypergeometric_2_f_1",
    "incomplete_beta",
    "log_beta",
    "log_gamma",
    "modified_bessel_i",
    "modified_bessel_i_0",
    "modified_bessel_i_1",
    "modified_bessel_k",
    "modified_bessel_k_0",
    "modified_bessel_k_1",
    "polygamma",
    "regularized_gamma_p",
    "regularized_gamma_q",
    "spherical_bessel_i",
    "spherical_bessel_i_0",
    "spherical_bessel_i_1",
    "spherical_bessel_j",
    "spherical_bessel_j_0",
    "spherical_bessel_j_1",
    "spherical_bessel_k",
    "spherical_bessel_k_0",
    "spherical_bessel_k_1",
    "spherical_bessel_y",
    "spherical_bessel_y_0",
    "spherical_bessel_y_1",
    "trigamma",
]
