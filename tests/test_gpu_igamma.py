"""Regularized incomplete gamma P/Q through the C ABI on the GPU: values against
scipy, parity with the reference, analytic derivatives against mpmath, mixed
against FP64, fused broadcast-reduced gradients, gradcheck/gradgradcheck."""

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden, rel_err, run

pytestmark = pytest.mark.gpu

D = golden("igamma")
A, X, G = D["a"], D["x"], D["g"]


def cuda(a, dtype=torch.float64):
    return torch.tensor(np.asarray(a), dtype=dtype, device="cuda")


def test_fp64_values_against_mpmath():
    """Relative error within 8 ulp x (1 + |ln value|) + 2e-14: the exponent
    a ln x - x - lnΓ(a) carries an absolute rounding error proportional to its
    size, which no double evaluation avoids (values down to e^-700 occur here);
    the 2e-14 floor covers the a < 10 branch, where the exponent is formed
    from terms of size ~20 directly."""
    (p,) = run("regularized_gamma_p", cuda(A), cuda(X))
    (q,) = run("regularized_gamma_q", cuda(A), cuda(X))
    p, q = p.cpu().numpy(), q.cpu().numpy()
    for got, tru in ((p, D["truth_p"]), (q, D["truth_q"])):
        m = tru > 1e-300
        bound = 8 * 2.2e-16 * (1 + np.abs(np.log(tru[m]))) + 2e-14
        e = rel_err(got, tru)[m]
        assert np.all(e <= bound), f"max rel err {e.max():.3e}, worst ratio {np.max(e / bound):.2f}"
    assert np.all(np.abs(p + q - 1) <= 8e-16)


def test_fp64_parity_with_reference():
    """|ours - ref| <= 4 ulp + |ref - truth| + our stated bound (the reference
    is accurate to ~1e-9 here: its series stops at 200 terms)."""
    (p,) = run("regularized_gamma_p", cuda(A), cuda(X))
    p = p.cpu().numpy()
    ref, tru = D["ref_regularized_gamma_p"], D["truth_p"]
    with np.errstate(divide="ignore"):
        ours = (8 * 2.2e-16 * (1 + np.abs(np.log(np.where(tru > 0, tru, 1.0)))) + 2e-14) * np.abs(tru)
    allowed = 4 * np.spacing(np.abs(ref)) + np.abs(ref - tru) + ours + 1e-300
    assert np.all(np.abs(p - ref) <= allowed)


def test_fp64_derivatives_against_mpmath():
    i = D["deriv_idx"]
    a, x = cuda(A[i]), cuda(X[i])
    one = torch.ones_like(a)
    ga, gx = run("regularized_gamma_p_backward", one, a, x, n_out=2)
    m = np.abs(D["truth_pa"]) > 1e-290
    e = rel_err(ga.cpu().numpy(), D["truth_pa"])[m]
    assert e.max() <= 1e-10, f"dP/da {e.max():.3e}"
    assert rel_err(gx.cpu().numpy(), D["truth_px"]).max() <= 1e-12
    # second derivatives through the double-backward entry point
    z = torch.zeros_like(a)
    o_g, o_a, o_x = run("regularized_gamma_p_backward_backward", one, z, one, a, x, n_out=3)  # gga=1, ggx=0
    m2 = np.abs(D["truth_paa"]) > 1e-280
    e2 = rel_err(o_a.cpu().numpy(), D["truth_paa"])[m2]
    assert np.median(e2) <= 1e-10 and e2.max() <= 1e-6, f"d2P/da2 {e2.max():.3e}"
    assert rel_err(o_x.cpu().numpy(), D["truth_pax"])[np.abs(D["truth_pax"]) > 1e-280].max() <= 1e-10
    _, _, o_xx = run("regularized_gamma_p_backward_backward", z, one, one, a, x, n_out=3)  # ggx=1
    assert rel_err(o_xx.cpu().numpy(), D["truth_pxx"])[np.abs(D["truth_pxx"]) > 1e-280].max() <= 1e-11


def test_q_derivatives_are_negated_p_derivatives():
    a, x, g = cuda(A), cuda(X), cuda(G)
    pa, px = run("regularized_gamma_p_backward", g, a, x, n_out=2)
    qa, qx = run("regularized_gamma_q_backward", g, a, x, n_out=2)
    assert torch.equal(pa, -qa) and torch.equal(px, -qx)


def test_mixed_within_1e6_of_fp64():
    a32, x32 = A.astype(np.float32), X.astype(np.float32)
    (pm,) = run("regularized_gamma_p", cuda(a32, torch.float32), cuda(x32, torch.float32))
    (pd,) = run("regularized_gamma_p", cuda(a32.astype(np.float64)), cuda(x32.astype(np.float64)))
    pm, pd = pm.cpu().numpy().astype(np.float64), pd.cpu().numpy()
    m = pd > 1e-30  # below float32's normal range the relative error is not meaningful
    e = rel_err(pm, pd)[m]
    assert e.max() <= 1e-6, f"mixed P {e.max():.3e}"
    g32 = G.astype(np.float32)
    gm = run("regularized_gamma_p_backward", cuda(g32, torch.float32), cuda(a32, torch.float32), cuda(x32, torch.float32), n_out=2)
    gd = run("regularized_gamma_p_backward", cuda(g32.astype(np.float64)), cuda(a32.astype(np.float64)), cuda(x32.astype(np.float64)), n_out=2)
    for k in range(2):
        u, v = gm[k].cpu().numpy().astype(np.float64), gd[k].cpu().numpy()
        mm = np.abs(v) > 1e-30
        e = rel_err(u, v)[mm]
        assert e.max() <= 1e-6, f"mixed grad {k}: {e.max():.3e}"


@pytest.mark.parametrize("upper", [False, True])
def test_mixed_within_1e6_of_fp64_on_the_broadcast_grid(upper):
    """Every element of a 1024 x 1024 grid of the benchmark distribution, as a
    broadcast (the per-row/column-table path) and element by element:
    P or Q and both derivatives, mixed against FP64 at the same float values."""
    gen = torch.Generator(device="cuda").manual_seed(3)
    lu = lambda shape, lo, hi: torch.exp(  # noqa: E731
        torch.rand(shape, generator=gen, device="cuda", dtype=torch.float64) * (np.log(hi) - np.log(lo)) + np.log(lo))
    a32, x32 = lu((1024, 1), 1e-2, 1e3).float(), lu((1, 1024), 1e-3, 2e3).float()
    name = "regularized_gamma_q" if upper else "regularized_gamma_p"
    g = torch.ones(1024, 1024, device="cuda")
    A32, X32 = a32.expand(1024, 1024).contiguous(), x32.expand(1024, 1024).contiguous()
    for aa, xx in ((a32, x32), (A32, X32)):
        (vm,) = run(name, aa, xx)
        (vd,) = run(name, aa.double(), xx.double())
        gm = run(name + "_backward", g, aa, xx, n_out=2)
        gd = run(name + "_backward", g.double(), aa.double(), xx.double(), n_out=2)
        for got, want in ((vm, vd), (gm[0], gd[0]), (gm[1], gd[1])):
            u, v = got.double().cpu().numpy(), want.cpu().numpy()
            m = (np.abs(v) > 1e-30) & (np.abs(v) < 3e38)
            e = rel_err(u, v)[m]
            assert e.max() <= 1e-6, f"{name}: {e.max():.3e}"


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_fused_reduced_gradients_match_full_gradients(dtype):
    """Config-2 broadcast layout (R,1) x (1,C): gradients reduced in-kernel
    (deterministic two-stage sum) equal the full-shape gradients summed."""
    gen = torch.Generator(device="cuda").manual_seed(0)
    R, C = 1000, 777
    a = torch.exp(torch.empty(R, 1, device="cuda", dtype=torch.float64).uniform_(np.log(1e-2), np.log(1e3), generator=gen)).to(dtype)
    x = torch.exp(torch.empty(1, C, device="cuda", dtype=torch.float64).uniform_(np.log(1e-3), np.log(2e3), generator=gen)).to(dtype)
    g = torch.randn(R, C, device="cuda", dtype=dtype, generator=gen)
    ga, gx = run("regularized_gamma_p_backward", g, a, x, n_out=2, out_shapes=[a.shape, x.shape])
    fa, fx = run("regularized_gamma_p_backward", g, a, x, n_out=2)
    ra = fa.double().sum(1, keepdim=True)
    rx = fx.double().sum(0, keepdim=True)
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    assert torch.allclose(ga.double(), ra, rtol=tol, atol=tol * ra.abs().max().item())
    assert torch.allclose(gx.double(), rx, rtol=tol, atol=tol * rx.abs().max().item())
    # deterministic: bitwise identical on a second call
    ga2, gx2 = run("regularized_gamma_p_backward", g, a, x, n_out=2, out_shapes=[a.shape, x.shape])
    assert torch.equal(ga, ga2) and torch.equal(gx, gx2)


def test_autograd_reduced_path_and_gradcheck():
    from torchscience_b200 import special_functions as sf

    gen = torch.Generator(device="cuda").manual_seed(1)
    a = (torch.rand(6, 1, device="cuda", dtype=torch.float64, generator=gen) * 5 + 0.2).requires_grad_()
    x = (torch.rand(1, 5, device="cuda", dtype=torch.float64, generator=gen) * 8 + 0.05).requires_grad_()
    y = sf.regularized_gamma_p(a, x)
    ga, gx = torch.autograd.grad(y.sum(), (a, x))
    fa, fx = run("regularized_gamma_p_backward", torch.ones(6, 5, device="cuda", dtype=torch.float64), a.detach(), x.detach(), n_out=2)
    assert torch.allclose(ga, fa.sum(1, keepdim=True), rtol=1e-13)
    assert torch.allclose(gx, fx.sum(0, keepdim=True), rtol=1e-13)
    assert torch.autograd.gradcheck(sf.regularized_gamma_p, (a, x), eps=1e-6, atol=1e-7, rtol=1e-5)
    assert torch.autograd.gradgradcheck(sf.regularized_gamma_p, (a, x), eps=1e-6, atol=1e-6, rtol=1e-4)
    assert torch.autograd.gradcheck(sf.regularized_gamma_q, (a, x), eps=1e-6, atol=1e-7, rtol=1e-5)


def test_full_size_properties_config2():
    """At the benchmark size (4096 x 4096 broadcast + 2^20 stress points):
    P + Q = 1, 0 <= P <= 1, and the recurrence P(a+1,x) = P(a,x) - x^a e^-x / Γ(a+1)."""
    from torchscience_b200 import special_functions as sf

    gen = torch.Generator(device="cuda").manual_seed(0)
    a = torch.exp(torch.empty(4096, 1, device="cuda", dtype=torch.float64).uniform_(np.log(1e-2), np.log(1e3), generator=gen))
    x = torch.exp(torch.empty(1, 4096, device="cuda", dtype=torch.float64).uniform_(np.log(1e-3), np.log(2e3), generator=gen))
    p = sf.regularized_gamma_p(a, x)
    q = sf.regularized_gamma_q(a, x)
    assert ((p + q - 1).abs().max().item()) <= 2e-15
    assert p.min().item() >= 0 and p.max().item() <= 1
    p1 = sf.regularized_gamma_p(a + 1, x)
    d = torch.exp(a * torch.log(x) - x - torch.lgamma(a + 1))
    r = (p1 - (p - d)).abs()
    assert r.max().item() <= 1e-12


def test_uniform_expansion_window_against_mpmath():
    """The transition window a >= 100, 0.6 <= x/a <= 1.6, evaluated by Temme's
    uniform expansion: P, Q (the smaller one directly), dP/da and dP/dx against
    mpmath at 50 digits, on a fixed grid of a (the window's edge 100 to 1e4)
    and x/a (both edges, x = a, and points on either side of the window, where
    the series and the continued fraction take over).  Bounds as in
    test_fp64_values_against_mpmath for the values, 1e-10 for dP/da, 1e-12 for
    dP/dx."""
    import mpmath

    a_list = [99.9, 100.0, 137.0, 273.0, 640.0, 1500.0, 4096.0, 1e4]
    lam_list = [0.55, 0.6, 0.61, 0.75, 0.9, 0.99, 1.0, 1.01, 1.2, 1.45, 1.59, 1.6, 1.7]
    a = np.array([av for av in a_list for _ in lam_list])
    x = np.array([av * lv for av in a_list for lv in lam_list])
    (p,) = run("regularized_gamma_p", cuda(a), cuda(x))
    (q,) = run("regularized_gamma_q", cuda(a), cuda(x))
    ga, gx = run("regularized_gamma_p_backward", cuda(np.ones_like(a)), cuda(a), cuda(x), n_out=2)
    p, q, ga, gx = [t.cpu().numpy() for t in (p, q, ga, gx)]
    with mpmath.workdps(50):
        _check_window(a, x, p, q, ga, gx)


def _check_window(a, x, p, q, ga, gx):
    import mpmath

    for i in range(a.size):
        am, xm = mpmath.mpf(a[i]), mpmath.mpf(x[i])
        tp = mpmath.gammainc(am, 0, xm, regularized=True)
        tq = mpmath.gammainc(am, xm, mpmath.inf, regularized=True)
        small, got = (tp, p[i]) if tp <= tq else (tq, q[i])
        if small < 1e-300:
            continue
        e = abs(got - float(small)) / float(small)
        bound = 8 * 2.2e-16 * (1 + abs(float(mpmath.log(small)))) + 2e-14
        assert e <= bound, f"a={a[i]} x={x[i]}: value rel err {e:.3e} > {bound:.3e}"
        # the derivative of the smaller function, so that 50 digits resolve it
        if tp <= tq:
            dpa = mpmath.diff(lambda s: mpmath.gammainc(s, 0, xm, regularized=True), am)
        else:
            dpa = -mpmath.diff(lambda s: mpmath.gammainc(s, xm, mpmath.inf, regularized=True), am)
        dpx = mpmath.exp((am - 1) * mpmath.log(xm) - xm - mpmath.loggamma(am))
        if abs(dpa) > 1e-290:
            ea = abs(ga[i] - float(dpa)) / abs(float(dpa))
            assert ea <= 1e-10, f"a={a[i]} x={x[i]}: dP/da rel err {ea:.3e}"
        if dpx > 1e-290:
            ex = abs(gx[i] - float(dpx)) / float(dpx)
            assert ex <= 1e-12, f"a={a[i]} x={x[i]}: dP/dx rel err {ex:.3e}"
