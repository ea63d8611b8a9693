"""log_beta, beta and polygamma through the C ABI on the GPU: values and
derivatives against mpmath (40 digits), including b << a where ψ(a) - ψ(a+b)
cancels and orders up to 30 of ψ^(n); parity with the reference where it is
accurate and closer-to-truth elsewhere; the reference's special points and
order conventions; float32 data; gradcheck and gradgradcheck."""

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden, rel_err, run
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu

D = golden("beta_family")
A, B, G = D["a"], D["b"], D["g"]
POS = (A > 0) & (B > 0)
EPS = np.finfo(np.float64).eps


def cuda(x, dtype=torch.float64):
    return torch.tensor(np.asarray(x), dtype=dtype, device="cuda")


def np_(t):
    return t.cpu().numpy().astype(np.float64)


# ------------------------------------------------------------------ log_beta
def test_log_beta_values():
    """Positive arguments: absolute error <= 4e-15 max(|ln B|, 1), from tiny to
    1e6 and with b down to 1e-12 a.  Negative a: the lnΓ sums, graded on the
    size of their terms."""
    (v,) = run("log_beta", cuda(A), cuda(B))
    v, t = np_(v), D["truth_lnb"]
    e = np.abs(v - t) / np.maximum(np.abs(t), 1.0)
    assert e[POS].max() <= 4e-15, f"positive: {e[POS].max():.3e}"
    from scipy.special import gammaln

    terms = np.abs(gammaln(A)) + np.abs(gammaln(B)) + np.abs(gammaln(A + B))
    en = np.abs(v - t) / np.maximum(terms, 1.0)
    assert en[~POS].max() <= 16 * EPS, f"negative: {en[~POS].max():.3e}"


def test_log_beta_gradients_without_cancellation():
    """ψ(a) - ψ(a+b) and ψ(b) - ψ(a+b) to <= 2e-15 relative for positive
    arguments (the reference's difference of ψ values is off by up to 1e-6
    relative when b << a)."""
    ga, gb = run("log_beta_backward", cuda(G), cuda(A), cuda(B), n_out=2)
    for got, tr, col in ((np_(ga), G * D["truth_da"], "da"), (np_(gb), G * D["truth_db"], "db")):
        e = rel_err(got, tr)
        assert e[POS].max() <= 2e-15, f"{col}: {e[POS].max():.3e}"
    ref = D["ref_log_beta_grad"][:, 0]
    tr = G * D["truth_da"]
    bad = POS & (rel_err(ref, tr) > 1e-10)
    assert bad.sum() > 20 and np.all(rel_err(np_(ga), tr)[bad] <= 2e-15)


def test_log_beta_double_backward():
    gga, ggb = D["gg"]
    o = run("log_beta_backward_backward", cuda(gga), cuda(ggb), cuda(G), cuda(A), cuda(B), n_out=3)
    o = [np_(t) for t in o]
    da, db, daa, dbb, dab = (D[f"truth_{k}"] for k in ("da", "db", "daa", "dbb", "dab"))
    want = [gga * da + ggb * db, G * (gga * daa + ggb * dab), G * (gga * dab + ggb * dbb)]
    scale = [np.abs(gga * da) + np.abs(ggb * db), np.abs(G) * (np.abs(gga * daa) + np.abs(ggb * dab)),
             np.abs(G) * (np.abs(gga * dab) + np.abs(ggb * dbb))]
    for got, w, sc in zip(o, want, scale):
        e = np.abs(got - w) / sc
        assert e[POS].max() <= 4e-15, f"{e[POS].max():.3e}"


# ---------------------------------------------------------------------- beta
def test_beta_values_and_signs():
    """B = exp(ln B) with relative error <= 4 ulp (1 + |ln B|) + 4e-15 where it
    is a normal number; negative a gives the signed value."""
    (v,) = run("beta", cuda(A), cuda(B))
    v, t = np_(v), D["truth_b"]
    m = (np.abs(t) > 1e-300) & (np.abs(t) < 1e300)
    bound = 4 * EPS * (1 + np.abs(D["truth_lnb"])) + 4e-15
    e = rel_err(v, t)
    assert np.all((e <= bound)[m & POS]), f"positive: {e[m & POS].max():.3e}"
    neg = m & ~POS
    assert np.all(np.sign(v[neg]) == np.sign(t[neg]))
    assert (np.sign(t[neg]) < 0).sum() > 20  # the sign matters in this sample
    from scipy.special import gammaln

    terms = np.abs(gammaln(A)) + np.abs(gammaln(B)) + np.abs(gammaln(A + B))
    assert np.all((e <= 8 * EPS * (1 + terms))[neg])


def test_beta_gradients():
    ga, gb = run("beta_backward", cuda(G), cuda(A), cuda(B), n_out=2)
    t, lb = D["truth_b"], D["truth_lnb"]
    m = POS & (np.abs(t) > 1e-290) & (np.abs(t) < 1e290)
    bound = 4 * EPS * (1 + np.abs(lb)) + 8e-15
    for got, d in ((np_(ga), D["truth_da"]), (np_(gb), D["truth_db"])):
        e = rel_err(got, G * t * d)
        assert np.all((e <= bound)[m]), f"{e[m].max():.3e}"


def test_beta_double_backward():
    gga, ggb = D["gg"]
    o = [np_(x) for x in run("beta_backward_backward", cuda(gga), cuda(ggb), cuda(G), cuda(A), cuda(B), n_out=3)]
    Bt = D["truth_b"]
    da, db, daa, dbb, dab = (D[f"truth_{k}"] for k in ("da", "db", "daa", "dbb", "dab"))
    haa, hab, hbb = Bt * (da * da + daa), Bt * (da * db + dab), Bt * (db * db + dbb)
    want = [Bt * (gga * da + ggb * db), G * (gga * haa + ggb * hab), G * (gga * hab + ggb * hbb)]
    scale = [np.abs(Bt) * (np.abs(gga * da) + np.abs(ggb * db)),
             np.abs(G * Bt) * (np.abs(gga) * (da * da + np.abs(daa)) + np.abs(ggb) * (np.abs(da * db) + np.abs(dab))),
             np.abs(G * Bt) * (np.abs(gga) * (np.abs(da * db) + np.abs(dab)) + np.abs(ggb) * (db * db + np.abs(dbb)))]
    m = POS & (np.abs(Bt) > 1e-290) & (np.abs(Bt) < 1e290)
    bound = 8 * EPS * (1 + np.abs(D["truth_lnb"])) + 1e-14
    for got, w, sc in zip(o, want, scale):
        e = np.abs(got - w) / sc
        assert np.all((e <= bound)[m]), f"{e[m].max():.3e}"


def test_parity_with_reference():
    """Where the reference is within 1e-12 of the truth, |ours - ref| <= 4 ulp +
    |ref - truth| + our bound; elsewhere ours is at least as close.  beta at
    negative arguments is graded on truth only: the reference drops the sign."""
    for op, t, scale in (("log_beta", D["truth_lnb"], np.maximum(np.abs(D["truth_lnb"]), 1.0)),
                         ("beta", D["truth_b"], np.abs(D["truth_b"]))):
        (v,) = run(op, cuda(A), cuda(B))
        v, ref = np_(v), D[f"ref_{op}"]
        fin = POS & np.isfinite(ref) & np.isfinite(t) & (scale > 1e-290) & (scale < 1e290)
        ours_e, ref_e = np.abs(v - t) / scale, np.abs(ref - t) / scale
        good = fin & (ref_e <= 1e-12)
        slack = 4 * EPS * (1 + np.abs(D["truth_lnb"])) + 4e-15
        assert np.all((np.abs(v - ref) <= 4 * np.spacing(np.abs(ref)) + np.abs(ref - t) + slack * scale)[good])
        assert np.all((ours_e <= ref_e + slack)[fin & ~good])


def test_reference_special_points():
    """(0, 1) and (-1, 1): poles of Γ(a) give +inf (the reference's tests require
    inf there); B(1, 1) = 1, B(1/2, 1/2) = π, B(2, 3) = 1/12; NaN propagates;
    B(3, 1e-300) = 1e300 within the bound of exp(ln B), 4 ulp (1 + |ln B|)."""
    sa, sb = D["special_a"], D["special_b"]
    (lb,) = run("log_beta", cuda(sa), cuda(sb))
    (bb,) = run("beta", cuda(sa), cuda(sb))
    lb, bb = np_(lb), np_(bb)
    assert np.isinf(lb[0]) and np.isinf(lb[1]) and np.isinf(bb[0])
    assert lb[2] == 0.0 and bb[2] == 1.0
    assert abs(bb[3] - np.pi) <= 2 * np.spacing(np.pi) and abs(bb[4] - 1 / 12) <= 4 * np.spacing(1 / 12)
    assert np.isnan(lb[5]) and np.isnan(lb[6]) and np.isnan(bb[5])
    assert lb[7] == -np.inf and bb[7] == 0.0
    assert bb[8] == pytest.approx(1e300, rel=4 * EPS * (1 + np.log(1e300)))


# ----------------------------------------------------------------- polygamma
PN, PZ, PG = D["pg_n"], D["pg_z"], D["pg_g"]


def pg_bound(v, dv):
    """1e-14 relative, or 8 ulp of the condition number |z ψ^(n+1)(z) / ψ^(n)(z)|
    where that is larger (negative z near the zeros and poles)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return 1e-14 + 8 * EPS * np.abs(PZ * dv / v)


def test_polygamma_values():
    """ψ^(n)(z) for n = 0..30, z in [1e-3, 1e3] and negative non-integer z:
    <= 1e-14 relative, or 8 ulp of the condition number where that is larger
    (the reference's n >= 4 series stops at about 1e-6 for small z).  Orders
    truncate toward zero as in the reference (2.7 -> 2, -0.5 -> 0); n <= -1
    and the poles give NaN (odd orders at a pole: +inf)."""
    (v,) = run("polygamma", cuda(PN), cuda(PZ))
    v, t = np_(v), D["pg_truth"]
    m = np.isfinite(t) & (np.abs(t) > 1e-300) & (np.abs(t) < 1e300)
    e = rel_err(v, t)
    b = pg_bound(t, D["pg_truth_d1"])
    assert np.all((e <= b)[m]), f"worst {(e / b)[m].max():.3e} of the bound"
    assert np.all(e[m & (PZ > 0)] <= 1e-14)
    assert np.median(e[m]) <= 2 * EPS
    tail = v[-9:]
    assert tail[0] == pytest.approx(t[-9], rel=1e-15) and tail[1] == pytest.approx(t[-8], rel=1e-15)
    assert np.isnan(tail[2]) and np.isnan(tail[3]) and tail[4] == np.inf
    ref = D["pg_ref"]
    hi = m & (PN >= 4) & (PZ > 0)
    assert rel_err(ref, t)[hi].max() > 1e-9  # the reference's truncation error ...
    assert np.all(e[hi] <= 1e-14)  # ... which ours does not have


def test_polygamma_backward_is_the_next_order():
    gn, gz = run("polygamma_backward", cuda(PG), cuda(PN), cuda(PZ), n_out=2)
    assert np.all(np_(gn) == 0)
    t = PG * D["pg_truth_d1"]
    m = np.isfinite(t) & (np.abs(t) > 1e-290) & (np.abs(t) < 1e290)
    b1 = pg_bound(D["pg_truth_d1"], D["pg_truth_d2"])
    assert np.all((rel_err(np_(gz), t) <= b1)[m])
    ggn, ggz = np.ones_like(PG), 0.5 * np.ones_like(PG)
    o = [np_(x) for x in run("polygamma_backward_backward", cuda(ggn), cuda(ggz), cuda(PG), cuda(PN), cuda(PZ), n_out=3)]
    w0, w2 = ggz * D["pg_truth_d1"], ggz * PG * D["pg_truth_d2"]
    m0 = np.isfinite(w0) & (np.abs(w0) > 1e-290) & (np.abs(w0) < 1e290)
    m2 = np.isfinite(w2) & (np.abs(w2) > 1e-290) & (np.abs(w2) < 1e290)
    assert np.all((rel_err(o[0], w0) <= b1)[m0]) and np.all(o[1] == 0)
    pos = m2 & (PZ > 0)
    assert rel_err(o[2], w2)[pos].max() <= 1e-14


# -------------------------------------------------------------------- common
@pytest.mark.parametrize("op", ["log_beta", "beta", "polygamma"])
def test_float32_data_is_the_fp64_value_rounded_once(op):
    x, y = (PN, PZ) if op == "polygamma" else (A, B)
    x32, y32 = x.astype(np.float32), y.astype(np.float32)
    (v32,) = run(op, cuda(x32, torch.float32), cuda(y32, torch.float32))
    (v64,) = run(op, cuda(x32.astype(np.float64)), cuda(y32.astype(np.float64)))
    assert torch.equal(v32.isnan(), v64.float().isnan())
    fin = ~v32.isnan()
    assert torch.equal(v32[fin], v64.float()[fin])


def test_gradcheck_and_gradgradcheck():
    gen = torch.Generator(device="cuda").manual_seed(7)
    a = (torch.rand(6, device="cuda", dtype=torch.float64, generator=gen) * 5 + 0.2).requires_grad_()
    b = (torch.rand(6, device="cuda", dtype=torch.float64, generator=gen) * 5 + 0.2).requires_grad_()
    for fn in (sf.log_beta, sf.beta):
        assert torch.autograd.gradcheck(fn, (a, b), eps=1e-6, atol=1e-7, rtol=1e-5)
        assert torch.autograd.gradgradcheck(fn, (a, b), eps=1e-6, atol=1e-6, rtol=1e-4)
    n = torch.tensor([0.0, 1.0, 2.0, 4.0, 5.0, 7.0], device="cuda", dtype=torch.float64)
    z = (torch.rand(6, device="cuda", dtype=torch.float64, generator=gen) * 5 + 0.5).requires_grad_()
    assert torch.autograd.gradcheck(lambda t: sf.polygamma(n, t), (z,), eps=1e-6, atol=1e-6, rtol=1e-5)
    assert torch.autograd.gradgradcheck(lambda t: sf.polygamma(n, t), (z,), eps=1e-6, atol=1e-5, rtol=1e-4)
