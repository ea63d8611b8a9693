"""The operators inside torch.compile (fullgraph): the compiled graph calls
them as opaque custom ops, with shapes from their Meta kernels and gradients
through their autograd registrations, and must reproduce eager results."""

import pytest
import torch

import torchscience_b200  # noqa: F401
from torchscience_b200 import probability as pb
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu


def _loss(a, x, z, m):
    p = sf.regularized_gamma_p(a, x)
    j = sf.bessel_j(torch.full_like(z, 1.5), z) + sf.bessel_j_0(z)
    k = sf.complete_legendre_elliptic_integral_k(m)
    lb = sf.log_beta(a, x)
    c = pb.gamma_cumulative_distribution(x, a, torch.ones_like(a))
    return (p * 2.0).sum() + (j * j).sum() + k.sum() + lb.sum() + c.sum()


def test_compiled_forward_and_backward_match_eager():
    torch._dynamo.reset()
    gen = torch.Generator(device="cuda").manual_seed(21)
    a = (torch.rand(64, 1, device="cuda", dtype=torch.float64, generator=gen) * 5 + 0.2).requires_grad_()
    x = (torch.rand(1, 48, device="cuda", dtype=torch.float64, generator=gen) * 8 + 0.1).requires_grad_()
    z = (torch.rand(100, device="cuda", dtype=torch.float64, generator=gen) * 20).requires_grad_()
    m = (torch.rand(100, device="cuda", dtype=torch.float64, generator=gen) * 0.9).requires_grad_()
    eager = _loss(a, x, z, m)
    ge = torch.autograd.grad(eager, (a, x, z, m))
    compiled = torch.compile(_loss, fullgraph=True)
    out = compiled(a, x, z, m)
    gc = torch.autograd.grad(out, (a, x, z, m))
    assert torch.allclose(out, eager, rtol=1e-13, atol=0)
    for u, v in zip(gc, ge):
        assert torch.allclose(u, v, rtol=1e-12, atol=1e-14)
