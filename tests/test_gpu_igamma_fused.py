"""The autograd path of regularized_gamma_p / _q when an input requires grad:
the forward evaluates P (Q) with its first derivatives in one pass and keeps
them, the backward multiplies them by the incoming gradient and reduces.  Its
gradients must equal the reference-named backward op's (which evaluates again
from the inputs), its forward value the plain forward's, and double backward
must keep working."""

import pytest
import torch

import torchscience_b200  # noqa: F401
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu

OPS = {"p": sf.regularized_gamma_p, "q": sf.regularized_gamma_q}


def inputs(shape_a, shape_x, dtype=torch.float64, seed=0):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    a = torch.exp(torch.rand(shape_a, device="cuda", dtype=torch.float64, generator=gen) * 11.5 - 4.6).to(dtype)
    x = torch.exp(torch.rand(shape_x, device="cuda", dtype=torch.float64, generator=gen) * 14.5 - 6.9).to(dtype)
    return a, x


def randn(shape, dtype, seed):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randn(shape, device="cuda", dtype=torch.float64, generator=gen).to(dtype)


def close(got, want, terms, tol, quantum=0.0):
    """|got - want| <= tol x (the sum of |terms| behind each reduced entry)
    + quantum x (the number of terms).  `want` and `terms` are the backward
    op's full-shape gradients (the reference's _backward ops return them
    unreduced), summed to got's shape.  `quantum` is the absolute rounding of
    one stored term: 0 for float64 data (the relative bound covers it); for
    float32 data the spacing of the subnormal floats, 2^-149, below which a
    float32 term has no relative precision left.  Returns (ok, report), the
    report naming the worst entry."""
    n_terms = want.numel() // got.numel()
    want, terms = want.double().sum_to_size(got.shape), terms.double().abs().sum_to_size(got.shape)
    err = (got.double() - want).abs()
    allowed = tol * terms + quantum * n_terms + 1e-300
    ratio = (err / allowed).flatten()
    k = int(torch.argmax(ratio))
    report = (f"worst |got - want| / allowed = {ratio[k].item():.3g} at flat index {k}: got "
              f"{got.double().flatten()[k].item():.6e}, want {want.flatten()[k].item():.6e}, "
              f"sum |terms| {terms.flatten()[k].item():.3e}")
    return bool((err <= allowed).all()), report


@pytest.mark.parametrize("which", ["p", "q"])
@pytest.mark.parametrize("layout", ["grid", "contiguous"])
def test_fused_gradients_equal_the_backward_op(which, layout):
    fn = OPS[which]
    if layout == "grid":
        a, x = inputs((384, 1), (1, 448))
    else:
        a, x = inputs((50000,), (50000,), seed=1)
        x = a * (1 + (x / x.max() - 0.5) * 2e-2)  # |x - a| < 1e-2 a, the benchmark's stress set
    g = randn(torch.broadcast_shapes(a.shape, x.shape), torch.float64, seed=10)
    ar, xr = a.clone().requires_grad_(True), x.clone().requires_grad_(True)
    y = fn(ar, xr)
    ga, gx = torch.autograd.grad(y, (ar, xr), g)
    with torch.no_grad():
        y0 = fn(a, x)
        ra, rx = getattr(torch.ops.torchscience, f"regularized_gamma_{which}_backward")(g, a, x)
        # per-entry scale of the reduction: the same reduction of |g·dP|
        ta, tx = getattr(torch.ops.torchscience, f"regularized_gamma_{which}_backward")(g.abs(), a, x)
    # the value comes from the derivative-carrying series / fraction, which may stop
    # a term later: equal to the plain forward within the evaluator's accuracy
    bound = 16 * 2.2e-16 * (1 + y0.abs().clamp_min(1e-300).log().abs()) * y0.abs()
    assert bool(((y - y0).abs() <= bound).all()), f"max |y - y0| / bound = {((y - y0).abs() / bound).max().item():.3g}"
    for got, want, terms in ((ga, ra, ta), (gx, rx, tx)):
        ok, report = close(got, want, terms, 1e-13)
        assert ok, report


@pytest.mark.parametrize("wants", ["a", "x"])
def test_one_input_requires_grad(wants):
    a, x = inputs((256, 1), (1, 320), seed=2)
    g = randn((256, 320), torch.float64, seed=11)
    ar = a.clone().requires_grad_(wants == "a")
    xr = x.clone().requires_grad_(wants == "x")
    y = sf.regularized_gamma_p(ar, xr)
    (gr,) = torch.autograd.grad(y, (ar if wants == "a" else xr,), g)
    with torch.no_grad():
        ra, rx = torch.ops.torchscience.regularized_gamma_p_backward(g, a, x)
        ta, tx = torch.ops.torchscience.regularized_gamma_p_backward(g.abs(), a, x)
    want, terms = (ra, ta) if wants == "a" else (rx, tx)
    ok, report = close(gr, want, terms, 1e-13)
    assert ok, report


@pytest.mark.parametrize("seed", [3, 4])
def test_float32_data(seed):
    """The kept derivatives of float32 data are float32 (rounded once each);
    the backward forms g x derivative in double and rounds the reduced sum
    once.  The _backward op rounds each full-shape product to float32.  Both
    agree to float32 accuracy relative to the size of the terms behind each
    reduced entry; where every term of an entry is a subnormal float32 (a
    column of x ~ 1.5e3 against a <= 1e3 has derivatives near 1e-42), the
    subnormal spacing 2^-149 is the only precision either side has."""
    a, x = inputs((256, 1), (1, 320), dtype=torch.float32, seed=seed)
    g = randn((256, 320), torch.float32, seed=12 + seed)
    ar, xr = a.clone().requires_grad_(True), x.clone().requires_grad_(True)
    ga, gx = torch.autograd.grad(sf.regularized_gamma_p(ar, xr), (ar, xr), g)
    with torch.no_grad():
        ra, rx = torch.ops.torchscience.regularized_gamma_p_backward(g, a, x)
        ta, tx = torch.ops.torchscience.regularized_gamma_p_backward(g.abs(), a, x)
    for got, want, terms in ((ga, ra, ta), (gx, rx, tx)):
        ok, report = close(got, want, terms, 2e-6, quantum=2.0**-149)
        assert ok, report


@pytest.mark.parametrize("which", ["p", "q"])
@pytest.mark.parametrize("layout", ["grid", "points"])
def test_float32_fused_forward_is_the_fp64_value_rounded_once(which, layout):
    """The fused forward evaluates float32 data with the FP64 evaluators and
    stores float32: its values equal the FP64 kernel's at the same inputs,
    rounded once, bit for bit, on the row-sorted sweep (grid) and on the map
    kernel (independent points at the transition x ~ a)."""
    if layout == "grid":
        a, x = inputs((192, 1), (1, 160), dtype=torch.float32, seed=21)
    else:
        a, _ = inputs((8192,), (1,), dtype=torch.float32, seed=22)
        x = (a.double() * (1.0 + (torch.rand(8192, device="cuda", dtype=torch.float64,
                                             generator=torch.Generator(device="cuda").manual_seed(23)) * 2 - 1)
                           * 1e-2)).float()
    ar, xr = a.clone().requires_grad_(True), x.clone().requires_grad_(True)
    y32 = OPS[which](ar, xr)
    y64 = OPS[which](a.double().requires_grad_(True), x.double().requires_grad_(True))
    assert y32.dtype == torch.float32
    assert torch.equal(y32.detach(), y64.detach().float())


def test_double_backward_through_the_fused_path():
    gen = torch.Generator(device="cuda").manual_seed(4)
    a = (torch.rand(5, 1, device="cuda", dtype=torch.float64, generator=gen) * 5 + 0.3).requires_grad_()
    x = (torch.rand(1, 4, device="cuda", dtype=torch.float64, generator=gen) * 6 + 0.2).requires_grad_()
    for fn in OPS.values():
        assert torch.autograd.gradcheck(fn, (a, x), eps=1e-6, atol=1e-7, rtol=1e-5)
        assert torch.autograd.gradgradcheck(fn, (a, x), eps=1e-6, atol=1e-6, rtol=1e-4)


def test_derivatives_are_kept_only_for_a_recorded_forward():
    """With grad enabled the forward keeps dP/da and dP/dx (two more tensors
    of the output's size stay alive with the graph); under no_grad the plain
    forward runs and only the output exists."""
    a, x = inputs((1024, 1), (1, 1024), seed=5)
    ar, xr = a.clone().requires_grad_(True), x.clone().requires_grad_(True)
    size = 1024 * 1024 * 8
    torch.cuda.synchronize()
    m0 = torch.cuda.memory_allocated()
    y = sf.regularized_gamma_p(ar, xr)
    kept = torch.cuda.memory_allocated() - m0
    del y
    with torch.no_grad():
        m1 = torch.cuda.memory_allocated()
        y = sf.regularized_gamma_p(ar, xr)
        plain = torch.cuda.memory_allocated() - m1
    assert kept >= 3 * size and plain < 2 * size


@pytest.mark.parametrize("layout", ["grid", "contiguous"])
def test_recompute_strategy(layout):
    """autograd_strategy("recompute"): the forward keeps nothing and the
    backward evaluates the derivatives again (reduced in the same pass); its
    gradients equal the kept-derivative ones."""
    if layout == "grid":
        a, x = inputs((300, 1), (1, 500), seed=6)
    else:
        a, x = inputs((40000,), (40000,), seed=7)
    g = randn(torch.broadcast_shapes(a.shape, x.shape), torch.float64, seed=13)
    grads = {}
    for strategy in ("keep", "recompute"):
        with torchscience_b200.autograd_strategy(strategy):
            ar, xr = a.clone().requires_grad_(True), x.clone().requires_grad_(True)
            torch.cuda.synchronize()
            m0 = torch.cuda.memory_allocated()
            y = sf.regularized_gamma_p(ar, xr)
            held = torch.cuda.memory_allocated() - m0
            grads[strategy] = torch.autograd.grad(y, (ar, xr), g)
            if strategy == "recompute":
                assert held < 2 * y.numel() * 8, held
    with torch.no_grad():
        ta, tx = torch.ops.torchscience.regularized_gamma_p_backward(g.abs(), a, x)
    for got, want, terms in zip(grads["recompute"], grads["keep"], (ta, tx)):
        scale = terms.double().abs().sum_to_size(got.shape)
        worst = ((got - want).abs() / (scale + 1e-300)).max().item()
        assert worst <= 1e-13, f"recompute vs keep: worst |difference| / sum |terms| = {worst:.3g}"
    assert torchscience_b200.get_autograd_strategy() == "keep"
