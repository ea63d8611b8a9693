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


def complete_legendre_elliptic_integral_e(m: Tensor) -> Tensor:
    """Complete elliptic integral of the second kind E(m) (parameter m = k²); NaN for m > 1, E(1) = 1.

    Same signature and semantics as the reference wrapper (src/torchscience/special_functions/_complete_legendre_elliptic_integral_e.py).
    """
    return torch.ops.torchscience.complete_legendre_elliptic_integral_e(m)


__all__ = ["complete_legendre_elliptic_integral_e", "complete_legendre_elliptic_integral_k", "digamma", "gamma", "log_gamma", "regularized_gamma_p", "regularized_gamma_q", "trigamma"]
