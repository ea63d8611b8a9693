"""Complex dtypes of log_beta and beta: values against mpmath (ln B as the sum
of principal lnΓ, as the reference's complex log_beta forms it, and B from
mpmath's beta), complex64 against complex128, broadcasting with reduced
gradients, and autograd's conjugate Wirtinger gradients (gradcheck /
gradgradcheck in complex128)."""

import mpmath
import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu


def points(n=400, seed=0):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-6, 12, n) + 1j * rng.uniform(-6, 6, n)
    b = rng.uniform(-6, 12, n) + 1j * rng.uniform(-6, 6, n)
    return a, b


def truth(a, b):
    with mpmath.workdps(40):
        lb = [complex(mpmath.loggamma(x) + mpmath.loggamma(y) - mpmath.loggamma(x + y)) for x, y in zip(a, b)]
        be = [complex(mpmath.beta(x, y)) for x, y in zip(a, b)]
    return np.array(lb), np.array(be)


def test_complex128_against_mpmath():
    a, b = points()
    ta, tb = (torch.tensor(v, device="cuda", dtype=torch.complex128) for v in (a, b))
    lb, be = sf.log_beta(ta, tb).cpu().numpy(), sf.beta(ta, tb).cpu().numpy()
    want_lb, want_be = truth(a, b)
    # ln B: each lnΓ carries ~1e-16 of its own size
    scale = np.abs(want_lb) + 10.0
    err = np.abs(lb - want_lb) / scale
    assert err.max() <= 1e-14, f"log_beta worst at a={a[np.argmax(err)]}, b={b[np.argmax(err)]}: {err.max():.2e}"
    # B = exp(ln B): the absolute rounding of ln B is B's relative error
    rel = np.abs(be - want_be) / np.abs(want_be)
    assert (rel <= 1e-14 * scale).all(), f"beta worst {rel.max():.2e}"


def test_complex64_against_complex128():
    a, b = points(seed=1)
    t64 = [torch.tensor(v, device="cuda", dtype=torch.complex64) for v in (a, b)]
    t128 = [t.to(torch.complex128) for t in t64]
    for fn in (sf.log_beta, sf.beta):
        lo, hi = fn(*t64).to(torch.complex128), fn(*t128)
        rel = ((lo - hi).abs() / hi.abs().clamp_min(1.0)).max().item()
        assert rel <= 5e-6, f"{fn.__name__}: {rel:.2e}"


@pytest.mark.parametrize("name", ["log_beta", "beta"])
def test_gradcheck_and_gradgradcheck_with_broadcasting(name):
    fn = getattr(sf, name)
    a = torch.tensor([[1.3 + 0.7j], [2.5 - 1.1j], [-3.4 + 0.6j]], device="cuda", dtype=torch.complex128,
                     requires_grad=True)
    b = torch.tensor([[0.4 + 2.2j, 3.0 - 0.5j, 1.7 + 0.1j, -0.6 - 1.3j]], device="cuda", dtype=torch.complex128,
                     requires_grad=True)
    assert torch.autograd.gradcheck(fn, (a, b), eps=1e-6, atol=1e-6, rtol=1e-5)
    assert torch.autograd.gradgradcheck(fn, (a, b), eps=1e-6, atol=1e-5, rtol=1e-4)
