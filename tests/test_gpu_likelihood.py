"""The Gamma log-likelihood workload through the public API on the GPU:
L = Σ[(k-1) ln x - x/θ - lnΓ(k) - k ln θ] with k ~ LogU(0.1, 100),
θ ~ LogU(0.1, 10), x ~ Gamma(k, scale θ); its gradients through autograd
(∂L/∂k = ln x - ψ(k) - ln θ, ∂L/∂θ = x/θ² - k/θ) and the Hessian-vector
product in k through double backward ((∇²_k L) v = -ψ'(k) v), in FP64 against
scipy and in FP32 against FP64."""

import math

import numpy as np
import pytest
import scipy.special as sp
import torch

import torchscience_b200  # noqa: F401
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu

N = 1 << 18


def inputs():
    gen = torch.Generator().manual_seed(0)

    def lu(lo, hi):
        u = torch.rand(N, generator=gen, dtype=torch.float64)
        return torch.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))

    k, theta = lu(0.1, 100.0), lu(0.1, 10.0)
    torch.manual_seed(0)
    x = torch.distributions.Gamma(k, 1.0 / theta).sample().clamp_min(1e-300)
    v = torch.randn(N, generator=torch.Generator().manual_seed(1), dtype=torch.float64)
    return k, theta, x, v


def loglik(k, theta, x):
    return ((k - 1) * torch.log(x) - x / theta - sf.log_gamma(k) - k * torch.log(theta)).sum()


def run_workload(dtype):
    k0, t0, x0, v0 = inputs()
    k = k0.to("cuda", dtype).requires_grad_()
    theta = t0.to("cuda", dtype).requires_grad_()
    x, v = x0.to("cuda", dtype), v0.to("cuda", dtype)
    L = loglik(k, theta, x)
    gk, gt = torch.autograd.grad(L, (k, theta), create_graph=True)
    (hvp,) = torch.autograd.grad(gk, k, v)
    return L.item(), gk.detach().double().cpu().numpy(), gt.detach().double().cpu().numpy(), hvp.double().cpu().numpy()


def test_fp64_gradients_and_hvp_against_scipy():
    k, theta, x, v = (t.numpy() for t in inputs())
    L, gk, gt, hvp = run_workload(torch.float64)
    want_L = np.sum((k - 1) * np.log(x) - x / theta - sp.gammaln(k) - k * np.log(theta))
    assert abs(L - want_L) <= 1e-12 * np.sum(np.abs((k - 1) * np.log(x)) + x / theta + np.abs(sp.gammaln(k)))
    want_gk = np.log(x) - sp.digamma(k) - np.log(theta)
    scale_k = np.abs(np.log(x)) + np.abs(sp.digamma(k)) + np.abs(np.log(theta))
    assert np.max(np.abs(gk - want_gk) / scale_k) <= 1e-14
    want_gt = x / theta**2 - k / theta
    assert np.max(np.abs(gt - want_gt) / (x / theta**2 + k / theta)) <= 1e-14
    want_h = -sp.polygamma(1, k) * v
    assert np.max(np.abs(hvp - want_h) / np.abs(want_h)) <= 1e-13


def test_fp32_within_1e6_of_fp64():
    k, theta, x, v = (t.numpy() for t in inputs())
    _, gk64, gt64, h64 = run_workload(torch.float64)
    _, gk32, gt32, h32 = run_workload(torch.float32)
    # FP32 inputs differ from FP64 ones by their rounding; compare the terms
    # each kernel owns: ψ(k) in ∂L/∂k and ψ'(k) in the HVP, relative to scale.
    scale_k = np.abs(np.log(x)) + np.abs(sp.digamma(k)) + np.abs(np.log(theta))
    k32 = k.astype(np.float32).astype(np.float64)
    x32, t32 = x.astype(np.float32).astype(np.float64), theta.astype(np.float32).astype(np.float64)
    ref_gk = np.log(x32) - sp.digamma(k32) - np.log(t32)
    assert np.max(np.abs(gk32 - ref_gk) / scale_k) <= 1e-6
    ref_h = -sp.polygamma(1, k32) * v.astype(np.float32).astype(np.float64)
    assert np.max(np.abs(h32 - ref_h) / np.abs(ref_h)) <= 1e-6
