"""The fused Gamma log-likelihood (value, gradient, Hessian-vector product):
FP64 against scipy, float32 against the FP64 kernels at the same values,
autograd (gradcheck / gradgradcheck), broadcasting and run-to-run
determinism of the sum."""

import numpy as np
import pytest
import scipy.special as sp
import scipy.stats as st
import torch

import torchscience_b200  # noqa: F401
from torchscience_b200 import probability as pr

pytestmark = pytest.mark.gpu


def sample(n, seed, dtype=torch.float64):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    lu = lambda lo, hi: torch.exp(  # noqa: E731
        torch.rand(n, generator=gen, device="cuda", dtype=torch.float64) * (np.log(hi) - np.log(lo)) + np.log(lo))
    k, th = lu(0.1, 100.0), lu(0.1, 10.0)
    torch.manual_seed(seed)
    x = torch.distributions.Gamma(k, 1.0 / th).sample().clamp_min(1e-30)
    return x.to(dtype), k.to(dtype), th.to(dtype)


def test_fp64_value_gradient_and_hvp_against_scipy():
    x, k, th = sample(1 << 16, 0)
    L, gx, gk, gt = pr.gamma_log_likelihood_value_and_grad(x, k, th, (True, True, True))
    xn, kn, tn = (t.cpu().numpy() for t in (x, k, th))
    ell = st.gamma.logpdf(xn, kn, scale=tn)
    want_L = np.sum(ell)
    assert abs(L.item() - want_L) <= 1e-12 * np.sum(np.abs(ell))
    want = {
        "x": (kn - 1) / xn - 1 / tn,
        "k": np.log(xn) - sp.digamma(kn) - np.log(tn),
        "t": xn / tn**2 - kn / tn,
    }
    for got, key in ((gx, "x"), (gk, "k"), (gt, "t")):
        w = want[key]
        scale = np.abs(w) + {"x": np.abs((kn - 1) / xn) + 1 / tn, "k": np.abs(np.log(xn)) + np.abs(sp.digamma(kn)) +
                             np.abs(np.log(tn)), "t": xn / tn**2 + kn / tn}[key]
        err = np.abs(got.cpu().numpy() - w) / scale
        assert err.max() <= 1e-13, (key, err.max())
    gen = torch.Generator(device="cuda").manual_seed(9)
    v = [torch.randn(x.shape, device="cuda", dtype=torch.float64, generator=gen) for _ in range(3)]
    hx, hk, ht = pr.gamma_log_likelihood_hvp(x, k, th, *v, grad=0.5)
    vn = [t.cpu().numpy() for t in v]
    H = [[-(kn - 1) / xn**2, 1 / xn, 1 / tn**2], [1 / xn, -sp.polygamma(1, kn), -1 / tn],
         [1 / tn**2, -1 / tn, kn / tn**2 - 2 * xn / tn**3]]
    for i, got in enumerate((hx, hk, ht)):
        terms = [H[i][j] * vn[j] for j in range(3)]
        w = 0.5 * sum(terms)
        err = np.abs(got.cpu().numpy() - w) / (0.5 * sum(np.abs(t) for t in terms))
        assert err.max() <= 1e-13, (i, err.max())


def test_float32_within_1e6_of_fp64():
    x, k, th = sample(1 << 20, 1)
    x32, k32, t32 = x.float(), k.float(), th.float()
    L32, _, gk32, gt32 = pr.gamma_log_likelihood_value_and_grad(x32, k32, t32, (False, True, True))
    L64, _, gk64, gt64 = pr.gamma_log_likelihood_value_and_grad(x32.double(), k32.double(), t32.double(),
                                                                (False, True, True))
    xn, kn, tn = (t.double().cpu().numpy() for t in (x32, k32, t32))
    ell_abs = np.abs((kn - 1) * np.log(xn)) + xn / tn + np.abs(sp.gammaln(kn)) + np.abs(kn * np.log(tn))
    assert abs(L32.item() - L64.item()) <= 1e-6 * ell_abs.sum()
    # gradients: relative to the size of the terms each is formed from
    sk = np.abs(np.log(xn)) + np.abs(sp.digamma(kn)) + np.abs(np.log(tn))
    st_ = xn / tn**2 + kn / tn
    for got, want, scale in ((gk32, gk64, sk), (gt32, gt64, st_)):
        err = np.abs(got.double().cpu().numpy() - want.cpu().numpy()) / scale
        assert err.max() <= 1e-6, err.max()
    v = torch.randn(x32.shape, device="cuda", generator=torch.Generator(device="cuda").manual_seed(4))
    (_, h32, _) = pr.gamma_log_likelihood_hvp(x32, k32, t32, None, v, None, out_mask=(False, True, False))
    (_, h64, _) = pr.gamma_log_likelihood_hvp(x32.double(), k32.double(), t32.double(), None, v.double(), None,
                                              out_mask=(False, True, False))
    err = ((h32.double() - h64).abs() / h64.abs().clamp_min(1e-30)).max().item()
    assert err <= 1e-6, err


def test_autograd_first_and_second_derivatives():
    gen = torch.Generator(device="cuda").manual_seed(5)
    x = (torch.rand(7, device="cuda", dtype=torch.float64, generator=gen) * 4 + 0.3).requires_grad_()
    k = (torch.rand(7, device="cuda", dtype=torch.float64, generator=gen) * 6 + 0.5).requires_grad_()
    th = (torch.rand(1, device="cuda", dtype=torch.float64, generator=gen) * 2 + 0.5).requires_grad_()  # broadcast
    assert torch.autograd.gradcheck(pr.gamma_log_likelihood, (x, k, th), eps=1e-6, atol=1e-8, rtol=1e-6)
    assert torch.autograd.gradgradcheck(pr.gamma_log_likelihood, (x, k, th), eps=1e-6, atol=1e-7, rtol=1e-5)


def test_hvp_through_autograd_equals_the_fused_op():
    x, k, th = sample(4096, 2)
    kr, tr = k.clone().requires_grad_(), th.clone().requires_grad_()
    L = pr.gamma_log_likelihood(x, kr, tr)
    gk, gt = torch.autograd.grad(L, (kr, tr), create_graph=True)
    v = torch.randn(k.shape, device="cuda", dtype=torch.float64, generator=torch.Generator(device="cuda").manual_seed(3))
    (hv,) = torch.autograd.grad(gk, kr, v)
    _, want, _ = pr.gamma_log_likelihood_hvp(x, k, th, None, v, None)
    assert torch.allclose(hv, want, rtol=1e-14, atol=0)
    assert torch.allclose(hv, -torch.special.polygamma(1, k) * v, rtol=1e-12)


def test_sum_is_deterministic_and_empty_is_zero():
    x, k, th = sample(3 << 20, 6)
    a = pr.gamma_log_likelihood_value_and_grad(x, k, th, (False, False, False))[0]
    b = pr.gamma_log_likelihood_value_and_grad(x, k, th, (False, False, False))[0]
    assert a.item() == b.item()
    e = torch.empty(0, device="cuda", dtype=torch.float64)
    assert pr.gamma_log_likelihood_value_and_grad(e, e, e, (False, False, False))[0].item() == 0.0
