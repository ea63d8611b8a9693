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
def test_a_series_past_its_cap_is_counted(dtype):
    # P(a, x) at a = x = 1e9 needs ~1e5 series terms; the cap is 2000
    a = torch.tensor([1e9, 2.0], device="cuda", dtype=dtype)
    x = torch.tensor([1e9, 1.0], device="cuda", dtype=dtype)
    tsb.unconverged_count(reset=True)
    p = sf.regularized_gamma_p(a, x)
    n = tsb.unconverged_count(reset=True)
    assert n == 1, n
    assert bool(torch.isfinite(p).all())
    assert tsb.unconverged_count() == 0  # the reset took effect


def test_check_convergence_warns_and_raises():
    a = torch.tensor([1e9], device="cuda", dtype=torch.float64)
    with pytest.warns(tsb.ConvergenceWarning):
        with tsb.check_convergence("warn"):
            sf.regularized_gamma_q(a, a)
    with pytest.raises(RuntimeError, match="iteration cap"):
        with tsb.check_convergence("raise"):
            sf.regularized_gamma_q(a, a)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        with tsb.check_convergence("warn"):
            sf.regularized_gamma_q(a * 0 + 3.0, a * 0 + 2.0)
