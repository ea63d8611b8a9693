"""Elements that stop at an iteration cap are counted (tsb_unconverged_count,
torchscience_b200.unconverged_count / check_convergence).  The loops are
bounded, so such inputs return a finite truncated value without hanging."""

import warnings

import pytest
import torch

import torchscience_b200 as tsb
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu


def test_ordinary_inputs_count_nothing():
    gen = torch.Generator(device="cuda").manual_seed(0)
    a = torch.exp(torch.rand(512, 1, device="cuda", dtype=torch.float64, generator=gen) * 11.5 - 4.6)
    x = torch.exp(torch.rand(1, 512, device="cuda", dtype=torch.float64, generator=gen) * 14.5 - 6.9)
    tsb.unconverged_count(reset=True)
    sf.regularized_gamma_p(a, x)
    sf.bessel_j(a.clamp_max(20), x)
    assert tsb.unconverged_count() == 0


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_a_fraction_past_its_cap_is_counted(dtype):
    # I_x(a, b) at x = 1/2, a = b = 1e9 needs ~2e4 terms of its continued
    # fraction next to the swap point; the cap is 4000 terms
    x = torch.tensor([0.5, 0.3], device="cuda", dtype=dtype)
    a = torch.tensor([1e9, 2.0], device="cuda", dtype=dtype)
    b = torch.tensor([1e9, 3.0], device="cuda", dtype=dtype)
    tsb.unconverged_count(reset=True)
    v = sf.incomplete_beta(x, a, b)
    n = tsb.unconverged_count(reset=True)
    assert n == 1, n
    assert bool(torch.isfinite(v).all())
    assert tsb.unconverged_count() == 0  # the reset took effect


def test_the_transition_at_large_a_reaches_no_cap():
    # P(a, x) at a = x = 1e9 would need ~1e5 series terms; the uniform
    # asymptotic expansion evaluates it in a fixed number of operations
    a = torch.tensor([1e9, 1e9 * 0.999, 1e9 * 1.001], device="cuda", dtype=torch.float64)
    tsb.unconverged_count(reset=True)
    p = sf.regularized_gamma_p(a.new_full((3,), 1e9), a)
    assert tsb.unconverged_count(reset=True) == 0
    assert bool(torch.isfinite(p).all())


def test_check_convergence_warns_and_raises():
    x = torch.tensor([0.5], device="cuda", dtype=torch.float64)
    a = torch.tensor([1e9], device="cuda", dtype=torch.float64)
    with pytest.warns(tsb.ConvergenceWarning):
        with tsb.check_convergence("warn"):
            sf.incomplete_beta(x, a, a)
    with pytest.raises(RuntimeError, match="iteration cap"):
        with tsb.check_convergence("raise"):
            sf.incomplete_beta(x, a, a)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        with tsb.check_convergence("warn"):
            sf.incomplete_beta(x * 0 + 0.3, a * 0 + 2.0, a * 0 + 3.0)
