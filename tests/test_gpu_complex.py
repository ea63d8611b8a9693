"""Complex dtypes of the gamma family (log_gamma, gamma, digamma, trigamma):
values against mpmath and against the reference's own complex outputs
(tests/golden/complex_gamma.npz, tests/golden/make_golden_complex.py),
complex64 against complex128, conjugate symmetry, and autograd's conjugate
Wirtinger gradients (gradcheck / gradgradcheck in complex128)."""

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu

OPS = {"log_gamma": sf.log_gamma, "gamma": sf.gamma, "digamma": sf.digamma, "trigamma": sf.trigamma}


def g():
    return golden("complex_gamma")


@pytest.mark.parametrize("name", list(OPS))
def test_complex128_against_mpmath(name):
    d = g()
    z = torch.tensor(d["z"], device="cuda", dtype=torch.complex128)
    got = OPS[name](z).cpu().numpy()
    want = d[f"truth_{name}"]
    ok = np.isfinite(want) & (np.abs(want) > 1e-300)
    if name == "gamma":
        # Γ = exp(lnΓ): the absolute rounding of lnΓ (~1e-16 |lnΓ|) is Γ's relative error
        tol = 1e-14 * np.maximum(1.0, np.abs(d["truth_log_gamma"]))
        err = np.abs(got - want) / np.abs(want)
    else:
        tol = 1e-14
        err = np.abs(got - want) / np.maximum(1.0, np.abs(want))
    bad = ok & ~(err <= tol)
    assert not bad.any(), f"{name}: {int(bad.sum())} points, worst z = {d['z'][ok][np.argmax(err[ok] / tol if np.ndim(tol) else err[ok])]}"


def test_log_gamma_matches_the_reference_up_to_its_branch():
    """The reference's complex log_gamma agrees with the principal branch in
    its real part; its imaginary part differs by multiples of 2π (a sum of
    principal logarithms).  So ours (the principal branch) matches it modulo
    2πi, and exp of both agree."""
    d = g()
    z = torch.tensor(d["z"], device="cuda", dtype=torch.complex128)
    got = sf.log_gamma(z).cpu().numpy()
    ref = d["ref_log_gamma"]
    ok = np.isfinite(ref)
    scale = np.maximum(1.0, np.abs(got))
    assert (np.abs(got.real - ref.real)[ok] <= 1e-12 * scale[ok]).all()
    k = (got.imag - ref.imag) / (2 * np.pi)
    assert (np.abs(k - np.round(k))[ok] * 2 * np.pi <= 1e-12 * scale[ok]).all()


@pytest.mark.parametrize("name", ["gamma", "digamma", "trigamma"])
def test_matches_the_reference_where_it_is_accurate(name):
    d = g()
    z = torch.tensor(d["z"], device="cuda", dtype=torch.complex128)
    got = OPS[name](z).cpu().numpy()
    ref, truth = d[f"ref_{name}"], d[f"truth_{name}"]
    ok = np.isfinite(ref) & np.isfinite(truth)
    rel = lambda u: np.abs(u - truth) / np.maximum(np.abs(truth), 1e-300)  # noqa: E731
    # ours is never farther from truth than the reference, beyond rounding
    # (for Γ = exp(lnΓ) that rounding is ~|lnΓ| ε relative)
    slack = 1e-14 * np.maximum(1.0, np.abs(d["truth_log_gamma"])) if name == "gamma" else 1e-13
    bad = ok & ~(rel(got) <= rel(ref) + slack)
    assert not bad.any(), f"{name}: {int(bad.sum())} points, e.g. z = {d['z'][bad][:3]}"


@pytest.mark.parametrize("name", list(OPS))
def test_complex64_and_conjugate_symmetry(name):
    d = g()
    z = torch.tensor(d["z"], device="cuda", dtype=torch.complex128)
    z64 = z.to(torch.complex64)
    lo = OPS[name](z64).to(torch.complex128)
    hi = OPS[name](z64.to(torch.complex128))
    fin = torch.isfinite(hi.real) & torch.isfinite(hi.imag) & (hi.abs() < 1e30) & (hi.abs() > 1e-30)
    rel = ((lo - hi).abs() / hi.abs().clamp_min(1.0 if name != "gamma" else 1e-300))[fin]
    assert rel.max().item() <= 2e-7
    a, b = OPS[name](z), OPS[name](z.conj()).conj()
    both = torch.isfinite(a.real) & torch.isfinite(b.real)
    assert torch.equal(a[both], b[both])


@pytest.mark.parametrize("name", list(OPS))
def test_gradcheck_and_gradgradcheck(name):
    z = torch.tensor([1.3 + 0.7j, 2.5 - 1.1j, -3.4 + 0.6j, 0.4 + 2.2j, -9.3 + 1.5j, 5.0 - 3.0j],
                     device="cuda", dtype=torch.complex128, requires_grad=True)
    fn = OPS[name]
    assert torch.autograd.gradcheck(fn, (z,), eps=1e-6, atol=1e-6, rtol=1e-5)
    assert torch.autograd.gradgradcheck(fn, (z,), eps=1e-6, atol=1e-5, rtol=1e-4)


def test_poles_and_specials():
    z = torch.tensor([0j, -1 + 0j, -7 + 0j, complex(float("nan"), 0)], device="cuda", dtype=torch.complex128)
    lg = sf.log_gamma(z).cpu()
    assert torch.isinf(lg.real[:3]).all() and (lg.imag[:3] == 0).all() and torch.isnan(lg.real[3])
    assert torch.isinf(sf.gamma(z).real[:3].cpu()).all()
    assert torch.isnan(sf.digamma(z).real[:3].cpu()).all()
