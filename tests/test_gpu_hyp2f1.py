"""Gauss 2F1(a, b; c; z) through the C ABI on the GPU: values, gradients and
Hessians against mpmath on a seeded sample of the benchmark distribution,
parity with the reference where it is accurate, the reference's own known
answers and special values, FP32 data against FP64, reduced (broadcast)
gradients, gradcheck and gradgradcheck."""

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import call, golden, rel_err, run
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu

D = golden("hyp2f1")
A, B, C, Z = D["a"], D["b"], D["c"], D["z"]
EPS = np.finfo(np.float64).eps
# Value bound: relative error <= 4096 ε (1 + κ), κ = Σ|x_i ∂F/∂x_i| / |F| the
# condition number of F in its inputs (ε κ is the error any FP64 method incurs
# from rounding the inputs; the factor absorbs the cancellation among series
# terms that κ does not see).
VALUE_FACTOR = 4096.0


def cuda(a, dtype=torch.float64):
    return torch.tensor(np.asarray(a), dtype=dtype, device="cuda")


def fwd(a, b, c, z, dtype=torch.float64):
    (v,) = run("hypergeometric_2_f_1", cuda(a, dtype), cuda(b, dtype), cuda(c, dtype), cuda(z, dtype))
    return v.cpu().numpy().astype(np.float64)


def grad(a, b, c, z, g=None):
    t = [cuda(v) for v in (a, b, c, z)]
    gt = cuda(np.ones(len(a)) if g is None else g)
    outs = run("hypergeometric_2_f_1_backward", gt, *t, n_out=4)
    return np.stack([o.cpu().numpy() for o in outs], axis=1)


def test_values_against_mpmath_within_condition_bound():
    v = fwd(A, B, C, Z)
    e = rel_err(v, D["truth"])
    bound = VALUE_FACTOR * EPS * (1.0 + D["kappa"])
    worst = np.argmax(e / bound)
    assert np.all(e <= bound), f"worst rel {e[worst]:.3e} at kappa {D['kappa'][worst]:.3e}"
    assert np.median(e) <= 2e-15
    assert np.quantile(e, 0.99) <= 1e-11


def test_parity_with_reference_where_it_is_accurate():
    """|ours - ref| <= 4 ulp + |ref - truth| + the value bound, on the points
    where the reference is within 1e-12 of mpmath (elsewhere, its unconverged
    series for z >= 1/2 and its cancellations, it is graded against truth only)."""
    v, ref, tru = fwd(A, B, C, Z), D["ref"], D["truth"]
    m = np.isfinite(ref) & (rel_err(ref, tru) <= 1e-12)
    assert m.mean() > 0.8
    allowed = 4 * np.spacing(np.abs(ref)) + np.abs(ref - tru) + VALUE_FACTOR * EPS * (1 + D["kappa"]) * np.abs(tru)
    assert np.all((np.abs(v - ref) <= allowed)[m])
    # Where it is not, ours is closer to mpmath: always inside the reference's
    # defect band (error > 1e-8), and on at least 90% of the remaining points
    # (the others are ill-conditioned ones where both sit at the rounding level).
    bad = ~m & np.isfinite(tru)
    closer = rel_err(v, tru) <= rel_err(ref, tru)
    assert np.all(closer[bad & (rel_err(ref, tru) > 1e-8)])
    assert closer[bad].mean() >= 0.9


def test_reference_known_answers_and_scipy_grid():
    k = D["kat"]
    v = fwd(*k[:, :4].T)
    finite = np.isfinite(k[:, 4])
    assert np.all(rel_err(v[finite], k[finite, 4]) <= 1e-10)
    assert np.all(np.isposinf(v[~finite]))
    g = D["grid"]
    assert rel_err(fwd(*g.T), D["grid_truth"]).max() <= 1e-13


def test_integer_c_minus_a_minus_b_near_one():
    """c - a - b (after Pfaff, a - b) an integer with the argument near 1: both
    terms of the connection formula are infinite; the shifted-c evaluation holds."""
    dg = D["degenerate"]
    assert rel_err(fwd(*dg.T), D["degenerate_truth"]).max() <= 1e-12


def test_special_values_match_reference():
    sp = D["special"]
    v = fwd(*sp.T)
    ref = D["special_ref"]
    assert np.array_equal(np.isnan(v), np.isnan(ref))
    assert np.array_equal(np.isinf(v), np.isinf(ref))
    fin = np.isfinite(ref)
    assert rel_err(v[fin], ref[fin]).max() <= 1e-14


def test_gradients_against_mpmath():
    G = grad(A, B, C, Z)
    T = D["truth_grad"]
    scale = np.abs(T).max(axis=1)
    e = np.abs(G - T).max(axis=1) / scale
    assert e.max() <= 2e-9, f"worst {e.max():.3e}"
    assert np.median(e) <= 1e-14


def test_gradients_match_reference_where_analytic():
    """The reference's parameter derivatives are analytic for |z| < 1/2 (its
    series; elsewhere finite differences with step 3e-8); dF/dz is analytic
    everywhere.  Where the reference's value is accurate, agree with it."""
    m = D["g"].size
    G = grad(A[:m], B[:m], C[:m], Z[:m], D["g"])
    R = D["ref_grad"]
    T = D["truth_grad"][:m] * D["g"][:, None]
    ok = (np.abs(Z[:m]) < 0.5) & np.isfinite(R).all(axis=1)
    scale = np.abs(T).max(axis=1)
    err_ours = np.abs(G - T).max(axis=1) / scale
    err_ref = np.abs(R - T).max(axis=1) / scale
    assert np.all((np.abs(G - R).max(axis=1) / scale <= err_ref + 1e-12 + err_ours)[ok])


def test_hessian_through_double_backward():
    n = D["truth_hess"].shape[0]
    t = [cuda(v[:n]) for v in (A, B, C, Z)]
    one = cuda(np.ones(n))
    H = np.empty((n, 4, 4))
    for j in range(4):
        gg = [cuda(np.full(n, float(i == j))) for i in range(4)]
        outs = run("hypergeometric_2_f_1_backward_backward", *gg, one, *t, n_out=5)
        for i in range(4):
            H[:, i, j] = outs[1 + i].cpu().numpy()
    pairs = [(0, 0), (0, 1), (0, 2), (0, 3), (1, 1), (1, 2), (1, 3), (2, 2), (2, 3), (3, 3)]
    got = np.stack([H[:, p, q] for p, q in pairs], axis=1)
    T = D["truth_hess"]
    e = np.abs(got - T).max(axis=1) / np.abs(T).max(axis=1)
    assert e.max() <= 1e-5, f"worst {e.max():.3e}"
    assert np.median(e) <= 1e-10
    assert np.allclose(H, np.transpose(H, (0, 2, 1)), rtol=1e-12, atol=0)


def test_fp32_data_matches_fp64_on_the_same_inputs():
    a32, b32, c32, z32 = (v.astype(np.float32) for v in (A, B, C, Z))
    v32 = fwd(a32, b32, c32, z32, torch.float32)
    v64 = fwd(a32.astype(np.float64), b32.astype(np.float64), c32.astype(np.float64), z32.astype(np.float64))
    m = np.isfinite(v64) & (np.abs(v64) < 3e38) & (np.abs(v64) > 1e-37)
    assert rel_err(v32[m], v64[m]).max() <= 1e-6


def test_broadcast_reduced_gradients_match_summed_full_gradients():
    dev = "cuda"
    gen = torch.Generator().manual_seed(7)
    a = (torch.rand(33, 1, generator=gen, dtype=torch.float64) * 6 - 3).to(dev).requires_grad_()
    b = (torch.rand(1, 29, generator=gen, dtype=torch.float64) * 6 - 3).to(dev).requires_grad_()
    c = torch.full((1, 1), 2.75, dtype=torch.float64, device=dev, requires_grad=True)
    z = (torch.rand(33, 29, generator=gen, dtype=torch.float64) * 5 - 4).to(dev).requires_grad_()
    y = sf.hypergeometric_2_f_1(a, b, c, z)
    g = torch.randn(y.shape, generator=gen, dtype=torch.float64).to(dev)
    ga, gb, gc, gz = torch.autograd.grad(y, (a, b, c, z), g)
    A_, B_, C_, Z_ = (t.detach().expand(33, 29).contiguous() for t in (a, b, c, z))
    full = torch.ops.torchscience.hypergeometric_2_f_1_backward(g, A_, B_, C_, Z_)
    torch.testing.assert_close(ga, full[0].sum(1, keepdim=True), rtol=1e-12, atol=1e-12)
    torch.testing.assert_close(gb, full[1].sum(0, keepdim=True), rtol=1e-12, atol=1e-12)
    torch.testing.assert_close(gc, full[2].sum().reshape(1, 1), rtol=1e-12, atol=1e-12)
    torch.testing.assert_close(gz, full[3], rtol=0, atol=0)


def test_gradcheck_and_gradgradcheck():
    dev = "cuda"
    a = torch.tensor([0.7, -1.3, 2.2, 3.1], dtype=torch.float64, device=dev, requires_grad=True)
    b = torch.tensor([1.4, 0.6, -2.5, 1.9], dtype=torch.float64, device=dev, requires_grad=True)
    c = torch.tensor([2.3, 3.6, 1.7, -1.5], dtype=torch.float64, device=dev, requires_grad=True)
    z = torch.tensor([0.3, -0.6, 0.8, -2.7], dtype=torch.float64, device=dev, requires_grad=True)
    assert torch.autograd.gradcheck(sf.hypergeometric_2_f_1, (a, b, c, z), eps=1e-6, atol=1e-7, rtol=1e-6)
    assert torch.autograd.gradgradcheck(sf.hypergeometric_2_f_1, (a, b, c, z), eps=1e-5, atol=1e-5, rtol=1e-4)


def test_grad_z_alone_matches_full_backward():
    """grad_z alone is (ab/c) 2F1(a+1, b+1; c+1; z) (one value evaluation);
    with the other grads it comes from the same pass as they do.  Both agree
    to the gradient bound."""
    t = [cuda(v[:500]) for v in (A, B, C, Z)]
    g = cuda(np.ones(500))
    gz = torch.empty_like(g)
    assert call("hypergeometric_2_f_1_backward", [g, *t], [None, None, None, gz]) == 0
    full = run("hypergeometric_2_f_1_backward", g, *t, n_out=4)[3]
    torch.testing.assert_close(gz, full, rtol=2e-9, atol=0)
