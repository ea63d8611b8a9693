"""incomplete_beta through the C ABI on the GPU: I_x(a, b), its first
derivatives and the six second derivatives against mpmath (40 digits) on
seeded x, a, b (next to the swap line x = (a+1)/(a+b+2), at a or b near 1,
for a, b up to 3000, and x within 1e-8 of 0 and 1); parity with the
reference where it is accurate and closer-to-truth elsewhere; the
reference's special points; float32 data; gradcheck and gradgradcheck."""

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden, rel_err, run
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu

D = golden("incomplete_beta")
X, A, B, G = D["x"], D["a"], D["b"], D["g"]
EPS = np.finfo(np.float64).eps
# Rounding of the exponent a ln x + b ln(1-x) - ln B(a, b) sets the error of
# every output: relative error of order ε (|a ln x| + |b ln(1-x)|).
BOUND = 16 * EPS * (1 + np.abs(A * np.log(X)) + np.abs(B * np.log1p(-X))) + 1e-15
# ∂a and ∂b also carry the rounding of K_p/K (or K_q/K) from the derivative
# recurrences of the continued fraction; next to the swap line, where K << 1
# and A_p/A, B_p/B nearly cancel, that is up to about 1.5e-12 relative.
DERIV_FLOOR = 4e-12


def cuda(x, dtype=torch.float64):
    return torch.tensor(np.asarray(x), dtype=dtype, device="cuda")


def np_(t):
    return t.cpu().numpy().astype(np.float64)


def test_values():
    (v,) = run("incomplete_beta", cuda(X), cuda(A), cuda(B))
    e = np.abs(np_(v) - D["truth_v"])
    assert np.all(e <= BOUND), f"worst {np.max(e / BOUND):.2f} x bound"


def test_values_parity_with_reference():
    """Within the reference's own error where it is accurate (its continued
    fraction stops at 200 terms, so for a, b in the thousands it is not)."""
    (v,) = run("incomplete_beta", cuda(X), cuda(A), cuda(B))
    v, ref, t = np_(v), D["ref"], D["truth_v"]
    ref_err = np.abs(ref - t)
    assert np.all(np.abs(v - ref) <= 4 * EPS + ref_err + BOUND)
    assert np.all(np.abs(v - t) <= np.maximum(ref_err, BOUND))


def test_first_derivatives():
    gx, ga, gb = run("incomplete_beta_backward", cuda(G), cuda(X), cuda(A), cuda(B), n_out=3)
    for got, col, tol in ((gx, "dx", 4 * BOUND), (ga, "da", np.maximum(4 * BOUND, DERIV_FLOOR)),
                          (gb, "db", np.maximum(4 * BOUND, DERIV_FLOOR))):
        e = rel_err(np_(got), G * D[f"truth_{col}"])
        assert np.all(e <= tol), f"{col}: worst {np.max(e / tol):.2f} x tolerance"


def test_parameter_derivatives_closer_than_reference():
    """The reference integrates log-weighted densities by adaptive quadrature
    (tolerance 1e-12, NaN at some points); where it is off by more than
    1e-10, ours is within the tolerance above."""
    _, ga, gb = run("incomplete_beta_backward", cuda(G), cuda(X), cuda(A), cuda(B), n_out=3)
    for got, col, k in ((ga, "da", 1), (gb, "db", 2)):
        tr = G * D[f"truth_{col}"]
        ref = D["ref_grad"][:, k]
        bad = ~(rel_err(ref, tr) <= 1e-10)
        assert bad.sum() > 50
        assert np.all(rel_err(np_(got), tr)[bad] <= np.maximum(4 * BOUND, DERIV_FLOOR)[bad])


def test_double_backward():
    """Second derivatives: x-x, x-a, x-b analytic, a-a, a-b, b-b central
    differences of the analytic first derivatives (step ε^(1/3)·a): each
    output within 1e-7 of the size of its terms."""
    i = D["idx2"]
    ggx, gga, ggb = (r[i] for r in D["gg"])
    g, x, a, b = G[i], X[i], A[i], B[i]
    o = run("incomplete_beta_backward_backward", cuda(ggx), cuda(gga), cuda(ggb), cuda(g), cuda(x), cuda(a), cuda(b),
            n_out=4)
    o = [np_(t) for t in o]
    t = {k: D[f"truth_{k}"] for k in ("hxx", "hxa", "hxb", "haa", "hab", "hbb")}
    dx, da, db = (D[f"truth_{k}"][i] for k in ("dx", "da", "db"))
    rows = [((ggx, dx), (gga, da), (ggb, db)),
            ((ggx, t["hxx"]), (gga, t["hxa"]), (ggb, t["hxb"])),
            ((ggx, t["hxa"]), (gga, t["haa"]), (ggb, t["hab"])),
            ((ggx, t["hxb"]), (gga, t["hab"]), (ggb, t["hbb"]))]
    for j, (got, terms) in enumerate(zip(o, rows)):
        mult = 1.0 if j == 0 else g
        want = mult * sum(u * v for u, v in terms)
        size = np.abs(mult) * sum(np.abs(u * v) for u, v in terms)
        tol = (np.maximum(4 * BOUND[i], DERIV_FLOOR) if j == 0 else 1e-7) * size + 1e-300
        assert np.all(np.abs(got - want) <= tol), f"output {j}: worst {np.max(np.abs(got - want) / tol):.2f}"


def test_special_points_match_reference():
    """NaN for a <= 0 or b <= 0 or NaN input, 0 / 1 outside (0, 1), the
    closed forms at a = 1 or b = 1; backward zeros outside (0, 1) (checked
    before the parameters), NaN for invalid parameters inside."""
    sx, sa, sb = D["special_x"], D["special_a"], D["special_b"]
    (v,) = run("incomplete_beta", cuda(sx), cuda(sa), cuda(sb))
    np.testing.assert_allclose(np_(v), D["special_ref"], rtol=1e-15, atol=0)
    g = run("incomplete_beta_backward", cuda(np.ones_like(sx)), cuda(sx), cuda(sa), cuda(sb), n_out=3)
    got = np.stack([np_(t) for t in g], axis=1)
    ref = D["special_ref_grad"]
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    fin = ~np.isnan(ref[:, 0])
    np.testing.assert_allclose(got[fin, 0], ref[fin, 0], rtol=1e-14, atol=1e-300)
    # the reference's a/b gradients are quadratures good to about 1e-7 here
    np.testing.assert_allclose(got[fin, 1:], ref[fin, 1:], rtol=1e-6, atol=1e-300)


def test_float32():
    (v,) = run("incomplete_beta", cuda(X, torch.float32), cuda(A, torch.float32), cuda(B, torch.float32))
    x32, a32, b32 = (np.float32(u).astype(np.float64) for u in (X, A, B))
    # evaluated in FP64 from the rounded inputs, rounded once: compare with the
    # FP64 op on the same rounded inputs
    (w,) = run("incomplete_beta", cuda(x32), cuda(a32), cuda(b32))
    want = np_(w).astype(np.float32).astype(np.float64)
    assert np.array_equal(np_(v), want)


def test_autograd_and_reduction():
    """Broadcast a and b: the gradients come back reduced to their shapes."""
    x = torch.rand(64, 8, dtype=torch.float64, device="cuda", requires_grad=True)
    a = (torch.rand(8, dtype=torch.float64, device="cuda") * 5 + 0.2).requires_grad_()
    b = (torch.rand(64, 1, dtype=torch.float64, device="cuda") * 5 + 0.2).requires_grad_()
    y = sf.incomplete_beta(x, a, b)
    gx, ga, gb = torch.autograd.grad(y.sum(), (x, a, b))
    assert gx.shape == x.shape and ga.shape == a.shape and gb.shape == b.shape
    full = run("incomplete_beta_backward", torch.ones_like(y), x.detach(), a.detach().expand_as(y),
               b.detach().expand_as(y), n_out=3)
    torch.testing.assert_close(ga, full[1].sum(0), rtol=1e-12, atol=1e-14)
    torch.testing.assert_close(gb, full[2].sum(1, keepdim=True), rtol=1e-12, atol=1e-14)


def test_gradcheck():
    torch.manual_seed(3)
    x = (torch.rand(6, dtype=torch.float64, device="cuda") * 0.8 + 0.1).requires_grad_()
    a = (torch.rand(6, dtype=torch.float64, device="cuda") * 4 + 0.5).requires_grad_()
    b = (torch.rand(6, dtype=torch.float64, device="cuda") * 4 + 0.5).requires_grad_()
    assert torch.autograd.gradcheck(sf.incomplete_beta, (x, a, b), eps=1e-6, atol=1e-7, rtol=1e-6)
    assert torch.autograd.gradgradcheck(sf.incomplete_beta, (x, a, b), eps=1e-6, atol=1e-6, rtol=1e-5)


def test_known_answers_from_reference_tests():
    """The reference's known answers (incomplete_beta_test.cpp:70-114,
    test__incomplete_beta.py:118-215): I_z(1, 1) = z, I_z(1, b) = 1 - (1-z)^b,
    I_z(a, 1) = z^a, I_z(a, b) + I_(1-z)(b, a) = 1, 0 at z = 0 and 1 at z = 1,
    at the reference's tolerances or tighter."""
    z = torch.tensor([0.0, 0.25, 0.5, 0.75, 1.0], dtype=torch.float64, device="cuda")
    one = torch.ones_like(z)
    torch.testing.assert_close(sf.incomplete_beta(z, one, one), z, rtol=0, atol=1e-15)
    z = torch.tensor([0.1, 0.25, 0.3, 0.5, 0.7, 0.75, 0.9], dtype=torch.float64, device="cuda")
    for v in (0.5, 2.0, 3.0, 7.5):
        c = torch.full_like(z, v)
        torch.testing.assert_close(sf.incomplete_beta(z, torch.ones_like(z), c), 1 - (1 - z) ** v, rtol=1e-14, atol=1e-15)
        torch.testing.assert_close(sf.incomplete_beta(z, c, torch.ones_like(z)), z**v, rtol=1e-14, atol=1e-15)
    for a, b in ((2.5, 3.5), (0.3, 12.0), (40.0, 0.7)):
        A, B = torch.full_like(z, a), torch.full_like(z, b)
        s = sf.incomplete_beta(z, A, B) + sf.incomplete_beta(1 - z, B, A)
        torch.testing.assert_close(s, torch.ones_like(z), rtol=0, atol=4e-16 * 4)
    for a, b in ((0.5, 0.5), (2.0, 3.0), (100.0, 0.1)):
        A = torch.full((2,), a, dtype=torch.float64, device="cuda")
        B = torch.full((2,), b, dtype=torch.float64, device="cuda")
        e = torch.tensor([0.0, 1.0], dtype=torch.float64, device="cuda")
        assert sf.incomplete_beta(e, A, B).tolist() == [0.0, 1.0]
