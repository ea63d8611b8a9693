"""Probability callers of the regularized incomplete gamma, with the reference's
Python API (torchscience.probability): the gamma, chi-squared and Poisson
cumulative distribution functions, the chi-squared survival function and the
gamma and chi-squared densities.  Each calls ``torch.ops.torchscience.<name>``,
registered for CUDA tensors by this package's native library; gradients come
from the ``<name>_backward`` operators (already reduced to the inputs' shapes).
"""

from __future__ import annotations

import torch
from torch import Tensor


def gamma_cumulative_distribution(x: Tensor, shape: Tensor, scale: Tensor) -> Tensor:
    """Gamma CDF F(x; shape, scale) = P(shape, x / scale); 0 for x <= 0.

    Same signature and semantics as the reference wrapper
    (src/torchscience/probability/_gamma/_gamma_cumulative_distribution.py).
    """
    return torch.ops.torchscience.gamma_cumulative_distribution(x, shape, scale)


def chi2_cumulative_distribution(x: Tensor, df: Tensor | float) -> Tensor:
    """Chi-squared CDF F(x; k) = P(k / 2, x / 2); 0 for x <= 0.

    Same signature and semantics as the reference wrapper
    (src/torchscience/probability/_chi2/_chi2_cumulative_distribution.py): a
    float ``df`` becomes a tensor of ``x``'s dtype and device.
    """
    return torch.ops.torchscience.chi2_cumulative_distribution(x, _df_tensor(x, df))


def poisson_cumulative_distribution(k: Tensor, rate: Tensor) -> Tensor:
    """Poisson CDF P(X <= k) = Q(floor(k) + 1, rate); 0 for k < 0; no gradient in k.

    Same signature and semantics as the reference wrapper
    (src/torchscience/probability/_poisson/_poisson_cumulative_distribution.py).
    """
    return torch.ops.torchscience.poisson_cumulative_distribution(k, rate)


def _df_tensor(x: Tensor, df: Tensor | float) -> Tensor:
    return df if isinstance(df, Tensor) else torch.as_tensor(df, dtype=x.dtype, device=x.device)


def chi2_survival(x: Tensor, df: Tensor | float) -> Tensor:
    """Chi-squared survival function 1 - F(x; k) = Q(k / 2, x / 2); 1 for x <= 0.

    Q is evaluated directly, so upper-tail values far below machine epsilon
    keep their relative accuracy.  Same signature and semantics as the
    reference wrapper (src/torchscience/probability/_chi2/_chi2_survival.py).
    """
    return torch.ops.torchscience.chi2_survival(x, _df_tensor(x, df))


def chi2_probability_density(x: Tensor, df: Tensor | float) -> Tensor:
    """Chi-squared density f(x; k) = x^(k/2-1) e^(-x/2) / (2^(k/2) Γ(k/2)).

    0 for x < 0; at x = 0: inf for k < 2, 1/2 for k = 2, 0 for k > 2.  Same
    signature and semantics as the reference wrapper
    (src/torchscience/probability/_chi2/_chi2_probability_density.py).
    """
    return torch.ops.torchscience.chi2_probability_density(x, _df_tensor(x, df))


def gamma_probability_density(x: Tensor, shape: Tensor, scale: Tensor) -> Tensor:
    """Gamma density f(x; shape, scale) = x^(shape-1) e^(-x/scale) / (scale^shape Γ(shape)); 0 for x <= 0.

    Same signature and semantics as the reference wrapper
    (src/torchscience/probability/_gamma/_gamma_probability_density.py).
    """
    return torch.ops.torchscience.gamma_probability_density(x, shape, scale)


__all__ = [
    "chi2_cumulative_distribution",
    "chi2_probability_density",
    "chi2_survival",
    "gamma_cumulative_distribution",
    "gamma_probability_density",
    "poisson_cumulative_distribution",
]
