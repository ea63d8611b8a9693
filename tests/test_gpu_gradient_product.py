"""The backward from kept derivatives (tsb_gradient_product through the C ABI):
g x d_a and g x d_x, each summed to its input's shape, against a float64
torch reference on ragged grids.  Double data runs the streaming 2-D kernel
(32-row x 256-column bands) when every operand is row-contiguous; float data
runs the tiled kernel.  Both must give the sums to the rounding of their
summation order, deterministically."""

import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import run

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (31, 257), (32, 256), (33, 255), (97, 1000), (1000, 97), (4096, 513)]
# the shapes of the two gradients: "row" = (rows, 1), "col" = (1, cols), "full" = (rows, cols)
LAYOUTS = [("row", "col"), ("col", "row"), ("row", "full"), ("full", "col")]


def out_shape(kind, rows, cols):
    return {"row": (rows, 1), "col": (1, cols), "full": (rows, cols)}[kind]


def sum_to(t, shape):
    dims = [d for d in range(2) if shape[d] == 1 and t.shape[d] != 1]
    return t.sum(dim=dims, keepdim=True) if dims else t


@pytest.mark.parametrize("rows,cols", SHAPES)
@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_reduced_products_against_torch(rows, cols, layout, dtype):
    gen = torch.Generator(device="cuda").manual_seed(rows * 7919 + cols)
    g, da, dx = (torch.randn(rows, cols, device="cuda", dtype=torch.float64, generator=gen).to(dtype) for _ in range(3))
    shapes = tuple(out_shape(k, rows, cols) for k in layout)
    ga, gx = run("gradient_product", g, da, dx, n_out=2, out_shapes=shapes)
    eps = 2.3e-16 if dtype == torch.float64 else 6e-8  # one rounding of the stored sum
    for got, d, shape in ((ga, da, shapes[0]), (gx, dx, shapes[1])):
        prod = g.double() * d.double()
        want, scale = sum_to(prod, shape), sum_to(prod.abs(), shape)
        assert got.shape == want.shape
        # double partial sums: a few units of 2^-53 times the sum of |terms|, then one rounding to the data type
        bound = 8 * 1.2e-16 * scale + eps * want.abs() + 1e-300
        err = (got.double() - want).abs()
        k = int(torch.argmax(err / bound))
        assert bool((err <= bound).all()), f"{shape}: worst entry {k}: {err.flatten()[k].item():.3e} > {bound.flatten()[k].item():.3e}"
    ga2, gx2 = run("gradient_product", g, da, dx, n_out=2, out_shapes=shapes)
    assert torch.equal(ga, ga2) and torch.equal(gx, gx2)  # deterministic
