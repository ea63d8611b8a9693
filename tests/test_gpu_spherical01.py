"""Spherical Bessel functions of order 0 and 1 as unary ops (j, y, i, k)
through the C ABI on the GPU: values, first and second derivatives against
the closed forms at 50 digits (mpmath), next to the zeros of j0, j1, y0, y1
too; parity with the reference; its special points; float32 data;
gradcheck and gradgradcheck."""

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden, run
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu

D = golden("spherical01")
OPS = [f"spherical_bessel_{k}_{n}" for k in "jyik" for n in (0, 1)]


def cuda(x, dtype=torch.float64):
    return torch.tensor(np.asarray(x), dtype=dtype, device="cuda")


def np_(t):
    return t.cpu().numpy().astype(np.float64)


def scale(name, z, t, q, t_next=None):
    """Error scale of derivative q: relative for i and k; for the oscillating j
    and y, floored at 1e-3 of the envelope (1/|z|)(1 + 1/|z|)^(q+n+1) and, next
    to a zero, at 1e-2 |z f^(q+1)(z)| (the condition number times |f|: the
    input's own rounding moves f by that much)."""
    if name[17] in "ik":
        return np.abs(t)
    n = int(name[-1])
    az = np.abs(z)
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        s = np.maximum(np.abs(t), 1e-3 / az * (1 + 1 / az) ** (q + n + 1))
        if t_next is not None:
            s = np.maximum(s, 1e-2 * az * np.abs(t_next))
    return s


TOL = (1e-14, 2e-14, 1e-13)  # value, first, second derivative


@pytest.mark.parametrize("name", OPS)
def test_values_and_derivatives(name):
    z, g, gg, t = D[f"{name}_z"], D[f"{name}_g"], D[f"{name}_gg"], D[f"{name}_truth"]
    (v,) = run(name, cuda(z))
    (gz,) = run(f"{name}_backward", cuda(g), cuda(z))
    ggo, gz2 = run(f"{name}_backward_backward", cuda(gg), cuda(g), cuda(z), n_out=2)
    for q, got, want, mult in ((0, np_(v), t[:, 0], 1.0), (1, np_(gz), t[:, 1], g), (1, np_(ggo), t[:, 1], gg),
                               (2, np_(gz2), t[:, 2], gg * g)):
        sc = scale(name, z, want, q, t[:, q + 1] if q < 2 else None) * np.abs(mult)
        m = np.isfinite(want) & np.isfinite(sc) & (sc > 1e-300) & (np.abs(want * mult) < 1e300)
        e = np.abs(got - mult * want) / sc
        assert e[m].max() <= TOL[q], f"{name} d{q}: worst {e[m].max():.3e} at z={z[m][np.argmax(e[m])]!r}"


@pytest.mark.parametrize("name", OPS)
def test_parity_with_reference(name):
    """Where the reference is within 1e-12 of the truth, |ours - ref| <= 4 ulp +
    |ref - truth| + our tolerance; elsewhere (its j1 = sin z/z² - cos z/z and
    i1 cancel for small |z|) ours is at least as close."""
    z, g, t = D[f"{name}_z"], D[f"{name}_g"], D[f"{name}_truth"]
    (v,) = run(name, cuda(z))
    (gz,) = run(f"{name}_backward", cuda(g), cuda(z))
    for q, got, ref, mult in ((0, np_(v), D[f"{name}_ref"], 1.0), (1, np_(gz), D[f"{name}_ref_grad"], g)):
        want = mult * t[:, q]
        sc = scale(name, z, t[:, q], q, t[:, q + 1]) * np.abs(mult)
        m = np.isfinite(want) & np.isfinite(ref) & (sc > 1e-300) & (np.abs(want) < 1e300)
        ours_e, ref_e = np.abs(got - want) / sc, np.abs(ref - want) / sc
        good = m & (ref_e <= 1e-12)
        allowed = 4 * np.spacing(np.abs(ref)) + np.abs(ref - want) + TOL[q] * sc
        assert np.all((np.abs(got - ref) <= allowed)[good])
        assert np.all((ours_e <= ref_e + TOL[q])[m & ~good])


@pytest.mark.parametrize("name", OPS)
def test_reference_special_points(name):
    """z = 0, -0, ±1e-13, -1, ±inf, NaN: the reference's values and first
    derivatives, except at ±inf, where the reference's closed forms give
    inf/inf or inf·0 = NaN and these return the limits (j, y, k: 0; i0: inf),
    and the y derivatives at ±0, which are NaN here."""
    sz = D[f"{name}_special_z"]
    (v,) = run(name, cuda(sz))
    (d,) = run(f"{name}_backward", cuda(np.ones_like(sz)), cuda(sz))
    v, d = np_(v), np_(d)
    rv, rd = D[f"{name}_special_ref"], D[f"{name}_special_ref_grad"]
    kind = name[17]
    keep = ~np.isinf(sz)
    assert np.allclose(v[keep], rv[keep], rtol=1e-14, atol=0, equal_nan=True), (v, rv)
    keep_d = keep & ~((sz == 0) & (kind == "y"))
    assert np.allclose(d[keep_d], rd[keep_d], rtol=1e-12, atol=0, equal_nan=True), (d, rd)
    if kind in "jy":
        assert np.all(v[np.isinf(sz)] == 0)
    if kind == "k":
        assert v[sz == np.inf][0] == 0
    if kind == "i" and name.endswith("0"):
        assert np.all(v[np.isinf(sz)] == np.inf)
    if kind == "y":
        assert np.all(np.isnan(d[sz == 0]))


@pytest.mark.parametrize("name", OPS)
def test_float32_data_is_the_fp64_value_rounded_once(name):
    z32 = D[f"{name}_z"].astype(np.float32)
    (v32,) = run(name, cuda(z32, torch.float32))
    (v64,) = run(name, cuda(z32.astype(np.float64)))
    assert torch.equal(v32.isnan(), v64.float().isnan())
    fin = ~v32.isnan()
    assert torch.equal(v32[fin], v64.float()[fin])


def test_gradcheck_and_gradgradcheck():
    gen = torch.Generator(device="cuda").manual_seed(17)
    z = (torch.rand(6, device="cuda", dtype=torch.float64, generator=gen) * 6 + 0.2).requires_grad_()
    for name in OPS:
        fn = getattr(sf, name)
        assert torch.autograd.gradcheck(fn, (z,), eps=1e-6, atol=1e-7, rtol=1e-5), name
        assert torch.autograd.gradgradcheck(fn, (z,), eps=1e-6, atol=1e-6, rtol=1e-4), name
