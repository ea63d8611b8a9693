"""The order-0/1 Bessel path through the C ABI on the GPU: J0 (bessel_j_0
forward, backward, double backward) and bessel_j at ν = 0, ±1, against
mpmath at 40 digits.  Below |x| = 16.25π the path keeps full relative
accuracy, next to the zeros too; above it the error is relative to the
envelope sqrt(J² + Y²).  Parity with the reference's bessel_j_0, FP32 data,
and the reference's special values."""

import numpy as np
import pytest
import scipy.special as sp
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden, run

pytestmark = pytest.mark.gpu

D = golden("bessel01")
X, G = D["x"], D["g"]
X0 = 16.25 * np.pi
SMALL = np.abs(X) < X0 * (1 - 1e-15)
TOL = 2e-15  # relative below X0, envelope-relative above
ENV0 = np.hypot(sp.j0(np.abs(X)), sp.y0(np.abs(X)))
ENV1 = np.hypot(sp.j1(np.abs(X)), sp.y1(np.abs(X)))


def cuda(a, dtype=torch.float64):
    return torch.tensor(np.asarray(a), dtype=dtype, device="cuda")


def scaled_err(got, want, env):
    """Relative error below X0 (including next to zeros), envelope-relative above."""
    scale = np.where(SMALL, np.abs(want), np.maximum(np.abs(want), env))
    return np.abs(got - want) / scale


def test_j0_forward_full_accuracy():
    (v,) = run("bessel_j_0", cuda(X))
    e = scaled_err(v.cpu().numpy(), D["truth_j0"], ENV0)
    assert e[SMALL].max() <= TOL, f"below X0: {e[SMALL].max():.3e}"
    assert e[~SMALL].max() <= TOL, f"above X0: {e[~SMALL].max():.3e}"
    assert np.median(e) <= 2e-16


def test_j0_backward_is_minus_j1():
    (gz,) = run("bessel_j_0_backward", cuda(G), cuda(X))
    want = -G * D["truth_j1"]
    m = D["truth_j1"] != 0
    e = scaled_err(gz.cpu().numpy(), want, np.abs(G) * ENV1)
    assert e[m].max() <= TOL + 1e-16, f"worst {e[m].max():.3e}"


def test_j0_double_backward():
    """{gg·J0'(x), gg·g·J0''(x)} with J0'' = J1/x - J0; at x = 0 J0'' = -1/2.
    J0'' is formed from J0 and J1, so it is graded relative to the envelope."""
    gg = np.full_like(X, 0.75)
    ggo, gz = run("bessel_j_0_backward_backward", cuda(gg), cuda(G), cuda(X), n_out=2)
    e1 = np.abs(ggo.cpu().numpy() + gg * D["truth_j1"]) / (np.abs(gg) * np.maximum(np.abs(D["truth_j1"]), ENV1))
    want2 = gg * G * D["truth_j0pp"]
    env2 = np.abs(gg * G) * np.maximum(np.abs(D["truth_j0pp"]), ENV0 + ENV1 / np.maximum(np.abs(X), 1e-300))
    e2 = np.abs(gz.cpu().numpy() - want2) / env2
    assert e1.max() <= 4e-15 and e2.max() <= 4e-15, (e1.max(), e2.max())
    a, b = run("bessel_j_0_backward_backward", cuda([1.0]), cuda([1.0]), cuda([0.0]), n_out=2)
    assert a.item() == 0.0 and b.item() == -0.5


@pytest.mark.parametrize("order", [0.0, 1.0, -1.0])
def test_bessel_j_at_orders_0_and_1_take_the_same_path(order):
    """bessel_j(ν, x) for ν = 0, ±1 and its x-derivative: J0' = -J1,
    J1' = J0 - J1/x, J_{-1} = -J_1."""
    n = np.full_like(X, order)
    (v,) = run("bessel_j", cuda(n), cuda(X))
    _, dz = run("bessel_j_backward", cuda(np.ones_like(X)), cuda(n), cuda(X), n_out=2)
    j0, j1 = D["truth_j0"], D["truth_j1"]
    if order == 0.0:
        tv, env, td, envd = j0, ENV0, -j1, ENV1
    else:
        s = np.sign(order)
        with np.errstate(divide="ignore", invalid="ignore"):
            d1 = np.where(X != 0, j0 - j1 / X, 0.5)
        tv, env, td, envd = s * j1, ENV1, s * d1, ENV0 + ENV1 / np.maximum(np.abs(X), 1e-300)
    m = tv != 0
    ev = scaled_err(v.cpu().numpy(), tv, env)
    assert ev[m].max() <= TOL, f"value {ev[m].max():.3e}"
    # the derivative truth for ν = ±1 is itself J0 - J1/x in float64: envelope-relative
    ed = np.abs(dz.cpu().numpy() - td) / np.maximum(np.abs(td), envd)
    assert ed[td != 0].max() <= 4e-15, f"derivative {ed[td != 0].max():.3e}"
    if order == 0.0:  # the same evaluator as bessel_j_0, up to the last rounding of the unrolled Horner
        (j0_op,) = run("bessel_j_0", cuda(X))
        assert np.all(np.abs(v.cpu().numpy() - j0_op.cpu().numpy()) <= 4 * np.spacing(np.abs(j0)))


def test_parity_with_reference_bessel_j_0():
    """|ours - ref| <= 4 ulp + |ref - truth| + 2e-15 of the local scale, and
    ours is never further from the truth than the reference by more than that
    scale: the reference's rational approximations lose accuracy next to
    zeros; ours do not."""
    (v,) = run("bessel_j_0", cuda(X))
    (gz,) = run("bessel_j_0_backward", cuda(G), cuda(X))
    for got, ref, tru, env in ((v.cpu().numpy(), D["ref_j0"], D["truth_j0"], ENV0),
                               (gz.cpu().numpy(), D["ref_j0_grad"], -G * D["truth_j1"], np.abs(G) * ENV1)):
        m = np.isfinite(ref)
        slack = TOL * np.maximum(np.abs(tru), env)
        allowed = 4 * np.spacing(np.abs(ref)) + np.abs(ref - tru) + slack
        assert np.all((np.abs(got - ref) <= allowed)[m])
        assert np.all((np.abs(got - tru) <= np.abs(ref - tru) + slack)[m])


def test_fp32_data_is_the_fp64_value_rounded_once():
    x32 = X.astype(np.float32)
    (v32,) = run("bessel_j_0", cuda(x32, torch.float32))
    (v64,) = run("bessel_j_0", cuda(x32.astype(np.float64)))
    assert torch.equal(v32, v64.float())
    g32 = G.astype(np.float32)
    (d32,) = run("bessel_j_0_backward", cuda(g32, torch.float32), cuda(x32, torch.float32))
    (d64,) = run("bessel_j_0_backward", cuda(g32.astype(np.float64)), cuda(x32.astype(np.float64)))
    assert torch.equal(d32, d64.float())


def test_special_values():
    (v,) = run("bessel_j_0", cuda([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, 1e300]))
    v = v.cpu().numpy()
    assert v[0] == 1 and v[1] == 1 and v[2] == 0 and v[3] == 0 and np.isnan(v[4]) and v[5] == 1
    assert abs(v[6]) <= 1e-150 and np.isfinite(v[6])
    (gz,) = run("bessel_j_0_backward", cuda([1.0, 1.0, 1.0]), cuda([0.0, np.inf, np.nan]))
    gz = gz.cpu().numpy()
    assert gz[0] == 0 and gz[1] == 0 and np.isnan(gz[2])
    (j,) = run("bessel_j", cuda([0.0, 1.0, -1.0, 1.0]), cuda([0.0, 0.0, np.inf, -2.0]))
    j = j.cpu().numpy()
    assert j[0] == 1 and j[1] == 0 and j[2] == 0 and j[3] == pytest.approx(-sp.j1(2.0), rel=1e-15)
