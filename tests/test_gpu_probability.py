"""Gamma, chi-squared and Poisson cumulative distributions (the probability
callers of P and Q) on the GPU: values against scipy, parity with the
reference's own kernels, gradients against closed forms and mpmath, the
reference's boundary conventions, broadcasting with reduced gradients."""

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden, rel_err
from torchscience_b200 import probability as pb

pytestmark = pytest.mark.gpu

D = golden("probability")
EPS = np.finfo(np.float64).eps


def cuda(a, dtype=torch.float64):
    return torch.tensor(np.asarray(a), dtype=dtype, device="cuda")


def bound(v):
    """Relative bound 16 ulp x (1 + |ln v|) + 5e-14: the incomplete gamma's
    (8 ulp x (1 + |ln v|) + 2e-14) with the rounding of the argument x/scale
    (x/2) and, for the Poisson CDF, of Q from the continued fraction."""
    with np.errstate(divide="ignore"):
        return 16 * EPS * (1 + np.abs(np.log(np.abs(v)))) + 5e-14


CASES = {
    "gamma": (lambda: pb.gamma_cumulative_distribution(cuda(D["gamma_x"]), cuda(D["gamma_shape"]), cuda(D["gamma_scale"]))),
    "chi2": (lambda: pb.chi2_cumulative_distribution(cuda(D["chi2_x"]), cuda(D["chi2_df"]))),
    "poisson": (lambda: pb.poisson_cumulative_distribution(cuda(D["poisson_k"]), cuda(D["poisson_rate"]))),
}


@pytest.mark.parametrize("name", list(CASES))
def test_values_against_scipy(name):
    v = CASES[name]().cpu().numpy()
    t = D[f"{name}_truth"]
    assert np.array_equal(np.isnan(v), np.isnan(t))
    m = np.isfinite(t) & (t > 1e-300)
    assert np.all((rel_err(v, t) <= bound(t))[m]), f"{name}: {rel_err(v, t)[m].max():.3e}"
    assert np.all(np.abs(v[t == 0]) < 1e-300)  # scipy underflows to 0 where ours is subnormal


@pytest.mark.parametrize("name", list(CASES))
def test_parity_with_reference_where_it_is_accurate(name):
    """|ours - ref| <= 4 ulp + |ref - truth| + the bound, where the reference is
    within 1e-12 of scipy; elsewhere (the Poisson CDF's Q = 1 - P cancellation
    for rate >> k) ours must be the closer one."""
    v = CASES[name]().cpu().numpy()
    ref, t = D[f"{name}_ref"], D[f"{name}_truth"]
    fin = np.isfinite(t) & np.isfinite(ref) & (np.abs(t) > 1e-300)
    good = fin & (rel_err(ref, t) <= 1e-12)
    allowed = 4 * np.spacing(np.abs(ref)) + np.abs(ref - t) + bound(t) * np.abs(t)
    assert np.all((np.abs(v - ref) <= allowed)[good])
    bad = fin & ~good
    assert np.all((rel_err(v, t) <= rel_err(ref, t))[bad])


def _grads(fn, inputs, g):
    ts = [cuda(a).requires_grad_(True) for a in inputs]
    y = fn(*ts)
    return [t.cpu().numpy() for t in torch.autograd.grad(y, ts, cuda(g))]


def test_gamma_gradients():
    x, sh, sc, g = D["gamma_x"], D["gamma_shape"], D["gamma_scale"], D["gamma_g"]
    gx, gs, gc = _grads(pb.gamma_cumulative_distribution, (x, sh, sc), g)
    pdf = D["gamma_truth_pdf"]
    m = np.isfinite(pdf) & (pdf > 1e-290)
    assert rel_err(gx, g * pdf)[m].max() <= 1e-12
    assert rel_err(gc, -g * pdf * x / sc)[m].max() <= 1e-12  # dF/dscale = -pdf x / scale
    i = D["gamma_dshape_idx"]
    tr = g[i] * D["gamma_truth_dshape"]
    mm = np.abs(tr) > 1e-290
    assert rel_err(gs[i], tr)[mm].max() <= 1e-9
    assert np.all(gx[x <= 0] == 0) and np.all(gs[x <= 0] == 0)


def test_chi2_gradients():
    x, df, g = D["chi2_x"], D["chi2_df"], D["chi2_g"]
    gx, gd = _grads(pb.chi2_cumulative_distribution, (x, df), g)
    pdf = D["chi2_truth_pdf"]
    m = np.isfinite(pdf) & (pdf > 1e-290)
    assert rel_err(gx, g * pdf)[m].max() <= 1e-12
    i = D["chi2_ddf_idx"]
    tr = g[i] * D["chi2_truth_ddf"]
    mm = np.abs(tr) > 1e-290
    assert rel_err(gd[i], tr)[mm].max() <= 1e-9


def test_poisson_gradients():
    k, r, g = D["poisson_k"], D["poisson_rate"], D["poisson_g"]
    gk, gr = _grads(pb.poisson_cumulative_distribution, (k, r), g)
    assert np.all(gk == 0)
    t = g * D["poisson_truth_drate"]
    m = np.isfinite(t) & (np.abs(t) > 1e-290)
    assert rel_err(gr, t)[m].max() <= 1e-12


def test_broadcast_and_reduced_gradients():
    x = cuda(np.linspace(0.1, 20.0, 64)).reshape(64, 1).requires_grad_(True)
    shape = cuda([0.5, 1.0, 2.5, 7.0]).reshape(1, 4).requires_grad_(True)
    scale = cuda([2.0]).requires_grad_(True)
    y = pb.gamma_cumulative_distribution(x, shape, scale)
    assert y.shape == (64, 4)
    gx, gs, gc = torch.autograd.grad(y.sum(), (x, shape, scale))
    assert gx.shape == x.shape and gs.shape == shape.shape and gc.shape == scale.shape
    full = torch.ops.torchscience.gamma_cumulative_distribution_backward(
        torch.ones(64, 4, dtype=torch.float64, device="cuda"), x.detach(), shape.detach(), scale.detach())
    torch.testing.assert_close(full[0], gx, rtol=0, atol=0)
    assert torch.autograd.gradcheck(
        pb.gamma_cumulative_distribution, (x[:8].detach().requires_grad_(), shape.detach().requires_grad_(),
                                           scale.detach().requires_grad_()))


def test_float32_within_1e6_of_float64():
    x, sh, sc = (D[f"gamma_{k}"][20:].astype(np.float32) for k in ("x", "shape", "scale"))
    v32 = pb.gamma_cumulative_distribution(*(cuda(a, torch.float32) for a in (x, sh, sc))).double().cpu().numpy()
    v64 = pb.gamma_cumulative_distribution(*(cuda(a.astype(np.float64)) for a in (x, sh, sc))).cpu().numpy()
    m = v64 > 1e-30
    assert rel_err(v32, v64)[m].max() <= 1e-6
