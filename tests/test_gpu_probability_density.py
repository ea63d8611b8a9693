"""Gamma and chi-squared densities and the chi-squared survival function on the
GPU: values and gradients against mpmath (40 digits), the reference's own
outputs at its boundary conventions, parity where the reference is accurate,
float32 data, broadcasting with reduced gradients, gradcheck."""

import numpy as np
import pytest
import scipy.special as sp
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden, rel_err
from torchscience_b200 import probability as pb

pytestmark = pytest.mark.gpu

D = golden("probability_density")
EPS = np.finfo(np.float64).eps


def cuda(a, dtype=torch.float64):
    return torch.tensor(np.asarray(a), dtype=dtype, device="cuda")


def density_bound(f, a, t):
    """Relative bound of a density value t^(a-1) e^(-t)/Γ(a): 16 ulp x (1 + |ln f|)
    for the exponent, 2 ulp x (|a - 1| + t) for the rounding of t = x/scale,
    and 5e-14."""
    with np.errstate(divide="ignore"):
        return 16 * EPS * (1 + np.abs(np.log(np.abs(f)))) + 2 * EPS * (np.abs(a - 1) + t) + 5e-14


def _grads(fn, inputs, g, dtype=torch.float64):
    ts = [cuda(a, dtype).requires_grad_(True) for a in inputs]
    y = fn(*ts)
    return [t.cpu().numpy().astype(np.float64) for t in torch.autograd.grad(y, ts, cuda(g, dtype))]


# ---------------------------------------------------------------- gamma density
GX, GA, GS, GG = D["gamma_x"], D["gamma_shape"], D["gamma_scale"], D["gamma_g"]
GT = GX / GS


def gamma_pdf(x=GX, a=GA, s=GS, dtype=torch.float64):
    return pb.gamma_probability_density(cuda(x, dtype), cuda(a, dtype), cuda(s, dtype)).cpu().numpy()


def test_gamma_density_values():
    v, t = gamma_pdf(), D["gamma_truth"]
    assert np.array_equal(np.isnan(v), np.isnan(t))
    m = np.isfinite(t) & (t > 1e-300)
    e = rel_err(v, t)
    assert np.all((e <= density_bound(t, GA, GT))[m]), f"worst {e[m].max():.3e}"
    assert np.median(e[m]) <= 2e-15
    assert np.all(np.abs(v[t == 0]) < 1e-300)


def test_gamma_density_gradients():
    gx, ga, gs = _grads(pb.gamma_probability_density, (GX, GA, GS), GG)
    tg = GG[:, None] * D["gamma_truth_grad"]
    f = np.abs(GG * D["gamma_truth"])
    m = np.isfinite(f) & (f > 1e-290)
    b = density_bound(D["gamma_truth"], GA, GT) + 1e-15
    # each derivative relative to the size of its factor's terms
    with np.errstate(divide="ignore", invalid="ignore"):
        scales = (f * (np.abs(GA - 1) + GT) / np.abs(GX), f * (np.abs(np.log(GT)) + np.abs(sp.digamma(GA))),
                  f * (GT + GA) / GS)
    for got, want, sc in zip((gx, ga, gs), tg.T, scales):
        err = np.abs(got - want) / sc
        assert np.all((err <= 4 * b)[m]), f"worst {np.nanmax(err[m]):.3e}"
    # x <= 0: zero gradients (the reference's convention)
    z = ~(GX > 0) & ~np.isnan(GX)
    assert np.all(gx[z] == 0) and np.all(ga[z] == 0) and np.all(gs[z] == 0)


def test_gamma_density_parity_with_reference():
    """Where the reference is within 1e-12 of the truth, |ours - ref| <= 4 ulp +
    |ref - truth| + our bound; elsewhere (its log-space formula loses digits for
    large shapes and arguments) ours is the closer one.  Boundary values match
    the reference exactly."""
    v, ref, t = gamma_pdf(), D["gamma_ref"], D["gamma_truth"]
    special = ~(GX > 0)
    assert np.array_equal(v[special], ref[special], equal_nan=True)
    fin = np.isfinite(t) & (t > 1e-300) & np.isfinite(ref)
    good = fin & (rel_err(ref, t) <= 1e-12)
    allowed = 4 * np.spacing(np.abs(ref)) + np.abs(ref - t) + density_bound(t, GA, GT) * t
    assert np.all((np.abs(v - ref) <= allowed)[good])
    assert np.all((rel_err(v, t) <= rel_err(ref, t) + density_bound(t, GA, GT))[fin & ~good])


def test_gamma_density_known_answers():
    """Exponential case (shape 1) and the reference test's scipy comparison point
    (shape 2, scale 2)."""
    x = np.array([0.5, 1.0, 2.0, 4.0])
    v = gamma_pdf(x, np.ones(4), np.full(4, 2.0))
    assert np.allclose(v, 0.5 * np.exp(-x / 2), rtol=4 * EPS, atol=0)
    v2 = gamma_pdf(x, np.full(4, 2.0), np.full(4, 2.0))
    assert np.allclose(v2, x * np.exp(-x / 2) / 4, rtol=8 * EPS, atol=0)


# ---------------------------------------------------------- chi-squared density
CX, CK, CG = D["chi2_x"], D["chi2_df"], D["chi2_g"]


def chi2_pdf(x=CX, k=CK, dtype=torch.float64):
    return pb.chi2_probability_density(cuda(x, dtype), cuda(k, dtype)).cpu().numpy()


def test_chi2_density_values_and_boundaries():
    v, t = chi2_pdf(), D["chi2_truth"]
    assert np.array_equal(np.isnan(v), np.isnan(t))
    # x = 0: inf for df < 2, 1/2 at df = 2, 0 above; x < 0: 0 (as the reference)
    assert v[0] == np.inf and v[1] == 0.5 and v[2] == 0 and v[3] == 0
    assert np.array_equal(v[:6], D["chi2_ref"][:6], equal_nan=True)
    m = np.isfinite(t) & (t > 1e-300) & (CX > 0)
    e = rel_err(v, t)
    assert np.all((e <= density_bound(t, CK / 2, CX / 2))[m]), f"worst {e[m].max():.3e}"


def test_chi2_density_gradients_and_parity():
    gx, gk = _grads(pb.chi2_probability_density, (CX, CK), CG)
    t = D["chi2_truth"]
    f = np.abs(CG * t)
    m = np.isfinite(f) & (f > 1e-290) & (CX > 0)
    b = density_bound(t, CK / 2, CX / 2) + 1e-15
    tg = CG[:, None] * D["chi2_truth_grad"]
    sx = f * (np.abs(CK / 2 - 1) + CX / 2) / np.maximum(CX, 1e-300)
    sk = f * (np.abs(np.log(np.maximum(CX, 1e-300) / 2)) + np.abs(sp.digamma(CK / 2))) / 2
    for got, want, sc in ((gx, tg[:, 0], sx), (gk, tg[:, 1], sk)):
        err = np.abs(got - want) / sc
        assert np.all((err <= 4 * b)[m]), f"worst {np.nanmax(err[m]):.3e}"
    # the reference's df-derivative is a central difference (step sqrt(eps)):
    # ours is at least as close to the truth, up to our bound
    ref = CG * D["chi2_ref_grad"][:, 1]
    fin = m & np.isfinite(ref)
    assert np.all((np.abs(gk - tg[:, 1]) <= np.abs(ref - tg[:, 1]) + 4 * b * sk)[fin])


# ---------------------------------------------------------- chi-squared survival
SX, SK, SG = D["sf_x"], D["sf_df"], D["sf_g"]


def chi2_sf(x=SX, k=SK, dtype=torch.float64):
    return pb.chi2_survival(cuda(x, dtype), cuda(k, dtype)).cpu().numpy()


def q_bound(v):
    with np.errstate(divide="ignore"):
        return 16 * EPS * (1 + np.abs(np.log(np.abs(v)))) + 5e-14


def test_chi2_survival_values():
    """Q is evaluated directly: the far upper tail keeps its relative accuracy
    (the reference forms it the same way, regularized_gamma_q)."""
    v, t = chi2_sf(), D["sf_truth"]
    assert np.array_equal(np.isnan(v), np.isnan(t))
    assert v[0] == 1 and v[1] == 1
    m = np.isfinite(t) & (t > 1e-300)
    e = rel_err(v, t)
    assert np.all((e <= q_bound(t))[m]), f"worst {e[m].max():.3e}"
    assert (t[m] < 1e-100).sum() > 10  # the tail is exercised


def test_chi2_survival_gradients_and_reference():
    gx, gk = _grads(pb.chi2_survival, (SX, SK), SG)
    tx = SG * D["sf_truth_dx"]
    m = np.isfinite(tx) & (np.abs(tx) > 1e-290)
    assert rel_err(gx, tx)[m].max() <= 1e-12
    i = D["sf_ddf_idx"]
    tk = SG[i] * D["sf_truth_ddf"]
    mm = np.abs(tk) > 1e-290
    assert rel_err(gk[i], tk)[mm].max() <= 1e-9
    v, ref, t = chi2_sf(), D["sf_ref"], D["sf_truth"]
    fin = np.isfinite(t) & np.isfinite(ref) & (t > 1e-300)
    good = fin & (rel_err(ref, t) <= 1e-12)
    allowed = 4 * np.spacing(np.abs(ref)) + np.abs(ref - t) + q_bound(t) * t
    assert np.all((np.abs(v - ref) <= allowed)[good])
    assert np.all((rel_err(v, t) <= rel_err(ref, t) + q_bound(t))[fin & ~good])


# ------------------------------------------------------------------- common
def test_float32_data_is_the_fp64_value_rounded_once():
    n = 512
    x32, a32, s32 = GX[:n].astype(np.float32), GA[:n].astype(np.float32), GS[:n].astype(np.float32)
    up = lambda a: a.astype(np.float64)  # noqa: E731
    assert np.array_equal(gamma_pdf(x32, a32, s32, torch.float32),
                          gamma_pdf(up(x32), up(a32), up(s32)).astype(np.float32), equal_nan=True)
    cx, ck = CX[:n].astype(np.float32), CK[:n].astype(np.float32)
    assert np.array_equal(chi2_pdf(cx, ck, torch.float32), chi2_pdf(up(cx), up(ck)).astype(np.float32), equal_nan=True)
    sx, sk = SX[:n].astype(np.float32), SK[:n].astype(np.float32)
    assert np.array_equal(chi2_sf(sx, sk, torch.float32), chi2_sf(up(sx), up(sk)).astype(np.float32), equal_nan=True)


@pytest.mark.parametrize("name", ["gamma_probability_density", "chi2_probability_density", "chi2_survival"])
def test_broadcast_reduced_gradients(name):
    """x (64, 1) against shape/df (1, 48): the backward op's gradients come back
    reduced to each input's shape and equal the sums of the expanded ones."""
    fn = getattr(pb, name)
    gen = torch.Generator(device="cuda").manual_seed(11)
    x = torch.rand(64, 1, device="cuda", dtype=torch.float64, generator=gen) * 20 + 0.05
    k = torch.rand(1, 48, device="cuda", dtype=torch.float64, generator=gen) * 10 + 0.3
    extra = [torch.rand(1, 48, device="cuda", dtype=torch.float64, generator=gen) + 0.5] if name.startswith("gamma") else []
    g = torch.randn(64, 48, device="cuda", dtype=torch.float64, generator=gen)
    ins = [x, k] + extra
    req = [t.clone().requires_grad_(True) for t in ins]
    grads = torch.autograd.grad(fn(*req), req, g)
    full = [t.expand(64, 48).clone().requires_grad_(True) for t in ins]
    gfull = torch.autograd.grad(fn(*full), full, g)
    for r, f, t in zip(grads, gfull, ins):
        assert r.shape == t.shape
        want = f.sum(dim=[d for d in range(2) if t.shape[d] == 1], keepdim=True)
        assert torch.allclose(r, want, rtol=1e-12, atol=1e-14)


def test_gradcheck():
    gen = torch.Generator(device="cuda").manual_seed(5)
    x = (torch.rand(6, device="cuda", dtype=torch.float64, generator=gen) * 5 + 0.2).requires_grad_()
    a = (torch.rand(6, device="cuda", dtype=torch.float64, generator=gen) * 4 + 0.5).requires_grad_()
    s = (torch.rand(6, device="cuda", dtype=torch.float64, generator=gen) * 2 + 0.5).requires_grad_()
    assert torch.autograd.gradcheck(pb.gamma_probability_density, (x, a, s), eps=1e-6, atol=1e-7, rtol=1e-5)
    assert torch.autograd.gradcheck(pb.chi2_probability_density, (x, a), eps=1e-6, atol=1e-7, rtol=1e-5)
    assert torch.autograd.gradcheck(pb.chi2_survival, (x, a), eps=1e-6, atol=1e-7, rtol=1e-5)
