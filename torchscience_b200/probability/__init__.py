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


# --------------------------------------------------------------------------
# Fused Gamma log-likelihood (an addition of this package: the reference
# builds it from log_gamma and elementwise ops).

def gamma_log_likelihood_value_and_grad(x: Tensor, shape: Tensor, scale: Tensor, grad_mask=(False, True, True)):
    """L = sum over elements of (shape - 1) ln x - x / scale - lnΓ(shape) - shape ln scale,
    and the per-element gradients dL/dx, dL/dshape, dL/dscale that `grad_mask`
    requests (None otherwise), from one pass over the inputs (one CUDA
    kernel plus the fixed-order sum of its block partials).  Returns
    (L, grad_x, grad_shape, grad_scale); the gradients have the broadcast
    shape of the inputs."""
    return torch.ops.torchscience_b200.gamma_log_likelihood_value_and_grad(x, shape, scale, list(grad_mask))


def gamma_log_likelihood_hvp(x: Tensor, shape: Tensor, scale: Tensor, v_x=None, v_shape=None, v_scale=None,
                             grad: Tensor | float = 1.0, out_mask=(True, True, True)):
    """Per element, grad · H v with H the Hessian of the log-density in (x, shape, scale):
        H = [[-(k-1)/x², 1/x, 1/θ²], [1/x, -ψ'(k), -1/θ], [1/θ², -1/θ, (k - 2x/θ)/θ²]].
    Any v may be None (zero).  Returns the three components (None where
    out_mask is False), each of the broadcast shape."""
    if not isinstance(grad, Tensor):
        grad = torch.tensor(grad, dtype=shape.dtype, device=shape.device)
    return torch.ops.torchscience_b200.gamma_log_likelihood_hvp(grad, x, shape, scale, v_x, v_shape, v_scale,
                                                                list(out_mask))


def _reduce_to(t, like):
    return None if t is None else t.sum_to_size(like.shape)


class _GammaLogLikelihood(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, shape, scale):
        mask = [bool(m) for m in ctx.needs_input_grad[:3]]
        value, gx, gk, gt = gamma_log_likelihood_value_and_grad(x, shape, scale, mask)
        ctx.save_for_backward(x, shape, scale, gx, gk, gt)
        return value

    @staticmethod
    def backward(ctx, g):
        x, k, th, gx, gk, gt = ctx.saved_tensors
        return _GammaLogLikelihoodBackward.apply(g, x, k, th, gx, gk, gt)


class _GammaLogLikelihoodBackward(torch.autograd.Function):
    """g times the per-element gradients kept by the forward, reduced to the
    inputs' shapes; its own backward is the Hessian-vector product."""

    @staticmethod
    def forward(ctx, g, x, k, th, gx, gk, gt):
        ctx.save_for_backward(g, x, k, th, gx, gk, gt)
        return tuple(None if d is None else _reduce_to(g * d, like) for d, like in ((gx, x), (gk, k), (gt, th)))

    @staticmethod
    def backward(ctx, ux, uk, ut):
        g, x, k, th, gx, gk, gt = ctx.saved_tensors
        want = [bool(m) for m in ctx.needs_input_grad[1:4]]
        hx = hk = ht = None
        if any(want):
            hx, hk, ht = gamma_log_likelihood_hvp(x, k, th, ux, uk, ut, grad=g, out_mask=want)
        gg = None
        if ctx.needs_input_grad[0]:
            gg = sum((u * d).sum() for u, d in ((ux, gx), (uk, gk), (ut, gt)) if u is not None and d is not None)
        return gg, _reduce_to(hx, x), _reduce_to(hk, k), _reduce_to(ht, th), None, None, None


def gamma_log_likelihood(x: Tensor, shape: Tensor, scale: Tensor) -> Tensor:
    """Sum of the Gamma(shape, scale) log-density over the broadcast elements
    of x, shape and scale, differentiable twice (the second derivative
    through the fused Hessian-vector product).  The forward evaluates the
    value and the requested first derivatives in one pass and keeps the
    derivatives for the backward."""
    return _GammaLogLikelihood.apply(x, shape, scale)
