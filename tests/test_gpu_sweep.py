"""The row-sorted sweep of (R, 1) x (1, C) grids (sweep.cuh) against the
unsorted tile kernel of the same entry point (called without the sweep's
scratch).  Both evaluate every element with the same functor and the same
per-row / per-column quantities, so full-shape outputs must be bit-identical;
reduced outputs are sums in another order and agree to 1e-13 of the sum of
the magnitudes of their terms."""

import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import run

pytestmark = pytest.mark.gpu


def grid(rows, cols, dtype, seed, transpose=False):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    a = torch.exp(torch.empty(rows, 1, device="cuda", dtype=torch.float64).uniform_(-4.6, 6.9, generator=gen))
    x = torch.exp(torch.empty(1, cols, device="cuda", dtype=torch.float64).uniform_(-6.9, 7.6, generator=gen))
    g = torch.randn(rows, cols, device="cuda", dtype=torch.float64, generator=gen)
    # edge values: a and x at 0, inf and NaN on a few rows / columns
    a[:3, 0] = torch.tensor([float("nan"), float("inf"), 1.0], device="cuda", dtype=torch.float64)
    x[0, :3] = torch.tensor([0.0, float("inf"), float("nan")], device="cuda", dtype=torch.float64)
    a, x, g = a.to(dtype), x.to(dtype), g.to(dtype)
    if transpose:
        a, x, g = a.t(), x.t(), g.t()
    return a, x, g


def same_bits(u, v):
    return bool(((u == v) | (torch.isnan(u) & torch.isnan(v))).all())


def close_sums(got, want, terms, tol=1e-13):
    got, want, terms = got.double(), want.double(), terms.double()
    finite = torch.isfinite(want)
    ok = (got - want).abs() <= tol * terms + 1e-300
    return bool((ok | ~finite).all()) and bool((torch.isnan(got) == torch.isnan(want)).all())


SHAPES = [(1000, 777), (4096, 64), (33, 5000), (64, 31)]


@pytest.mark.parametrize("rows,cols", SHAPES)
@pytest.mark.parametrize("transpose", [False, True])
@pytest.mark.parametrize("which", ["p", "q"])
def test_forward_and_forward_with_grads_bit_identical(rows, cols, transpose, which):
    a, x, _ = grid(rows, cols, torch.float64, seed=rows + cols, transpose=transpose)
    name = f"regularized_gamma_{which}"
    (y_sw,) = run(name, a, x)
    (y_tile,) = run(name, a, x, sweep=False)
    assert same_bits(y_sw, y_tile)
    fg_sw = run(f"{name}_forward_with_grads", a, x, n_out=3)
    fg_tile = run(f"{name}_forward_with_grads", a, x, n_out=3, sweep=False)
    for u, v in zip(fg_sw, fg_tile):
        assert same_bits(u, v)


@pytest.mark.parametrize("rows,cols", SHAPES)
@pytest.mark.parametrize("transpose", [False, True])
def test_backward_reduced_and_full(rows, cols, transpose):
    a, x, g = grid(rows, cols, torch.float64, seed=7 + rows, transpose=transpose)
    name = "regularized_gamma_p_backward"
    full_sw = run(name, g, a, x, n_out=2)
    full_tile = run(name, g, a, x, n_out=2, sweep=False)
    for u, v in zip(full_sw, full_tile):
        assert same_bits(u, v)
    red_sw = run(name, g, a, x, n_out=2, out_shapes=[a.shape, x.shape])
    red_tile = run(name, g, a, x, n_out=2, out_shapes=[a.shape, x.shape], sweep=False)
    terms = run(name, g.abs(), a, x, n_out=2)
    for got, want, full, t in zip(red_sw, red_tile, full_sw, terms):
        shape = got.shape
        assert close_sums(got, want, t.abs().sum_to_size(shape))
        assert close_sums(got, full.sum_to_size(shape), t.abs().sum_to_size(shape))


def test_double_backward_three_output_kinds():
    """_backward_backward on the grid: one full output (the gradient of the
    incoming gradient) and two reduced ones, in one sweep."""
    a, x, g = grid(513, 300, torch.float64, seed=11)
    gen = torch.Generator(device="cuda").manual_seed(12)
    gga = torch.randn(a.shape, device="cuda", dtype=torch.float64, generator=gen)
    ggx = torch.randn(x.shape, device="cuda", dtype=torch.float64, generator=gen)
    name = "regularized_gamma_p_backward_backward"
    shapes = [g.shape, a.shape, x.shape]
    sw = run(name, gga, ggx, g, a, x, n_out=3, out_shapes=shapes)
    tile = run(name, gga, ggx, g, a, x, n_out=3, out_shapes=shapes, sweep=False)
    full = run(name, gga, ggx, g, a, x, n_out=3)
    terms = run(name, gga.abs(), ggx.abs(), g.abs(), a, x, n_out=3)
    # the same kernel with other output kinds: identical.  The tile kernel is
    # another instantiation of the second-order evaluator, and its row and
    # column tables (lnΓ, ψ, ψ' of a, ln x) come from its own compiled code
    # rather than the sweep's set-up kernel; either may round a sum of
    # products differently in the last place, which the second-order loop's
    # stopping rule (a term later or sooner) carries into dP/da: equal to 64
    # ulp of |gga dP/da| + |ggx dP/dx| (measured: 25).
    assert same_bits(sw[0], full[0])
    assert bool((torch.isnan(sw[0]) == torch.isnan(tile[0])).all())
    da, dx = run("regularized_gamma_p_backward", torch.ones_like(g), a, x, n_out=2)
    fin = torch.isfinite(tile[0])
    diff = (sw[0] - tile[0]).abs()[fin]
    scale = (gga.abs() * da.abs() + ggx.abs() * dx.abs())[fin]
    worst = (diff / (scale + 1e-300)).max().item()
    assert worst <= 64 * 2.2e-16, f"sweep vs tile, double backward: {worst:.3g} of the terms"
    for k in (1, 2):
        scale = terms[k].abs().sum_to_size(shapes[k])
        assert close_sums(sw[k], tile[k], scale) and close_sums(sw[k], full[k].sum_to_size(shapes[k]), scale)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16])
def test_low_precision_storage(dtype):
    a, x, g = grid(700, 450, dtype, seed=3)
    (y_sw,) = run("regularized_gamma_p", a, x)
    (y_tile,) = run("regularized_gamma_p", a, x, sweep=False)
    assert same_bits(y_sw, y_tile)
    fg_sw = run("regularized_gamma_p_forward_with_grads", a, x, n_out=3)
    fg_tile = run("regularized_gamma_p_forward_with_grads", a, x, n_out=3, sweep=False)
    for u, v in zip(fg_sw, fg_tile):
        assert same_bits(u, v)


def test_deterministic_reductions():
    a, x, g = grid(2048, 1024, torch.float64, seed=5)
    r1 = run("regularized_gamma_p_backward", g, a, x, n_out=2, out_shapes=[a.shape, x.shape])
    r2 = run("regularized_gamma_p_backward", g, a, x, n_out=2, out_shapes=[a.shape, x.shape])
    for u, v in zip(r1, r2):
        assert same_bits(u, v)
