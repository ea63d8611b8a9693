"""Probability callers of the regularized incomplete gamma, with the reference's
Python API (torchscience.probability): the gamma, chi-squared and Poisson
cumulative distribution functions.  Each calls ``torch.ops.torchscience.<name>``,
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
    df_t = df if isinstance(df, Tensor) else torch.as_tensor(df, dtype=x.dtype, device=x.device)
    return torch.ops.torchscience.chi2_cumulative_distribution(x, df_t)


def poisson_cumulative_distribution(k: Tensor, rate: Tensor) -> Tensor:
    """Poisson CDF P(X <= k) = Q(floor(k) + 1, rate); 0 for k < 0; no gradient in k.

    Same signature and semantics as the reference wrapper
    (src/torchscience/probability/_poisson/_poisson_cumulative_distribution.py).
    """
    return torch.ops.torchscience.poisson_cumulative_distribution(k, rate)


__all__ = [
    "chi2_cumulative_distribution",
    "gamma_cumulative_distribution",
    "poisson_cumulative_distribution",
]
