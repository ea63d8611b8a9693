"""Integer-order Bessel functions as unary ops (bessel_j_1, bessel_y_0,
bessel_y_1, modified_bessel_i_0/_1, modified_bessel_k_0/_1) through the C ABI
on the GPU: values, first and second derivatives against mpmath (40 digits),
next to the zeros of J1, Y0, Y1 too; parity with the reference; its special
points; float32 data; gradcheck and gradgradcheck."""

import numpy as np
import pytest
import scipy.special as sp
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden, run
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu

D = golden("bessel_int")
OPS = ["bessel_j_1", "bessel_y_0", "bessel_y_1", "modified_bessel_i_0", "modified_bessel_i_1",
       "modified_bessel_k_0", "modified_bessel_k_1"]
ORDER = {n: int(n[-1]) for n in OPS}
X0 = 16.25 * np.pi


def cuda(x, dtype=torch.float64):
    return torch.tensor(np.asarray(x), dtype=dtype, device="cuda")


def np_(t):
    return t.cpu().numpy().astype(np.float64)


def scales(name, z, t):
    """Per-point error scales of (f, f', f'').  J and Y oscillate: below 16.25π
    J1 is graded relative to itself (the order-0/1 path keeps relative accuracy
    at its zeros) and J1' = J0 - J1/z on the size of those two terms; Y and
    large-z J relative to the envelope sqrt(J² + Y²) of the order (and of the
    next order for f').  I and K do not vanish: relative.
    f'' comes from Bessel's equation, so it is graded on the size of its terms
    |f'|/|z| + (1 + ν²/z²)|f|."""
    az = np.abs(z)
    n = ORDER[name]
    with np.errstate(all="ignore"):
        if name.startswith("bessel"):
            env = np.hypot(sp.jv(n, az), sp.yv(n, az))
            env1 = np.hypot(sp.jv(n + 1, az), sp.yv(n + 1, az)) + env / np.maximum(az, 1e-300)
            s0 = np.maximum(np.abs(t[:, 0]), env if name != "bessel_j_1" else np.where(az < X0, 0.0, env))
            # J1' = J0 - J1/z: below X0 graded on the size of those terms
            terms = np.abs(sp.j0(az)) + np.abs(sp.j1(az)) / np.maximum(az, 1e-300)
            s1 = np.maximum(np.abs(t[:, 1]), env1 if name != "bessel_j_1" else np.where(az < X0, terms, env1))
        else:
            s0, s1 = np.abs(t[:, 0]), np.abs(t[:, 1])
        s2 = np.maximum(np.abs(t[:, 2]), s1 / np.maximum(az, 1e-300) + (1 + n * n / np.maximum(az * az, 1e-300)) * s0)
    return s0, s1, s2


TOL = {"bessel_j_1": 2e-15, "bessel_y_0": 3e-14, "bessel_y_1": 3e-14, "modified_bessel_i_0": 1e-14,
       "modified_bessel_i_1": 1e-14, "modified_bessel_k_0": 1e-14, "modified_bessel_k_1": 1e-14}


def _usable(t, sc):
    return np.isfinite(t) & np.isfinite(sc) & (sc > 1e-300) & (sc < 1e300)


@pytest.mark.parametrize("name", OPS)
def test_values_and_derivatives(name):
    z, g, gg = D[f"{name}_z"], D[f"{name}_g"], D[f"{name}_gg"]
    t = D[f"{name}_truth"]
    s0, s1, s2 = scales(name, z, t)
    (v,) = run(name, cuda(z))
    (gz,) = run(f"{name}_backward", cuda(g), cuda(z))
    ggo, gz2 = run(f"{name}_backward_backward", cuda(gg), cuda(g), cuda(z), n_out=2)
    for label, got, want, sc in (("f", np_(v), t[:, 0], s0), ("f'", np_(gz), g * t[:, 1], np.abs(g) * s1),
                                 ("f' (bb)", np_(ggo), gg * t[:, 1], np.abs(gg) * s1),
                                 ("f''", np_(gz2), gg * g * t[:, 2], np.abs(gg * g) * s2)):
        m = _usable(want, sc)
        e = np.abs(got - want) / sc
        tol = TOL[name] * (4 if label == "f''" else (2 if label != "f" else 1))
        assert e[m].max() <= tol, f"{name} {label}: worst {e[m].max():.3e} at z={z[m][np.argmax(e[m])]!r}"


@pytest.mark.parametrize("name", OPS)
def test_parity_with_reference(name):
    """Where the reference is within 1e-12 of the truth (on the scales above),
    |ours - ref| <= 4 ulp + |ref - truth| + our tolerance; elsewhere ours is at
    least as close."""
    z, g = D[f"{name}_z"], D[f"{name}_g"]
    t = D[f"{name}_truth"]
    s0, s1, _ = scales(name, z, t)
    (v,) = run(name, cuda(z))
    (gz,) = run(f"{name}_backward", cuda(g), cuda(z))
    for got, ref, want, sc in ((np_(v), D[f"{name}_ref"], t[:, 0], s0),
                               (np_(gz), D[f"{name}_ref_grad"], g * t[:, 1], np.abs(g) * s1)):
        m = _usable(want, sc) & np.isfinite(ref)
        ours_e, ref_e = np.abs(got - want) / sc, np.abs(ref - want) / sc
        good = m & (ref_e <= 1e-12)
        allowed = 4 * np.spacing(np.abs(ref)) + np.abs(ref - want) + 2 * TOL[name] * sc
        assert np.all((np.abs(got - ref) <= allowed)[good])
        assert np.all((ours_e <= ref_e + 2 * TOL[name])[m & ~good])


@pytest.mark.parametrize("name", OPS)
def test_reference_special_points(name):
    """z = 0, -0, -1, ±inf, NaN, 1e-13: the reference's values and first
    derivatives (to rounding at -1 and 1e-13), except I1'(±inf), which is +inf here (the reference's
    I0 - I1/z forms inf - inf)."""
    sz = D[f"{name}_special_z"]
    (v,) = run(name, cuda(sz))
    (d,) = run(f"{name}_backward", cuda(np.ones_like(sz)), cuda(sz))
    v, d = np_(v), np_(d)
    rv, rd = D[f"{name}_special_ref"], D[f"{name}_special_ref_grad"]
    keep = ~((name == "modified_bessel_i_1") & np.isinf(sz))
    assert np.allclose(v, rv, rtol=1e-14, atol=0, equal_nan=True), (v, rv)
    assert np.allclose(d[keep], rd[keep], rtol=1e-12, atol=0, equal_nan=True), (d, rd)


@pytest.mark.parametrize("name", OPS)
def test_float32_data_is_the_fp64_value_rounded_once(name):
    z32 = D[f"{name}_z"].astype(np.float32)
    (v32,) = run(name, cuda(z32, torch.float32))
    (v64,) = run(name, cuda(z32.astype(np.float64)))
    assert torch.equal(v32.isnan(), v64.float().isnan())
    fin = ~v32.isnan()
    assert torch.equal(v32[fin], v64.float()[fin])


def test_gradcheck_and_gradgradcheck():
    gen = torch.Generator(device="cuda").manual_seed(13)
    z = (torch.rand(6, device="cuda", dtype=torch.float64, generator=gen) * 8 + 0.3).requires_grad_()
    for name in OPS:
        fn = getattr(sf, name)
        assert torch.autograd.gradcheck(fn, (z,), eps=1e-6, atol=1e-7, rtol=1e-5), name
        assert torch.autograd.gradgradcheck(fn, (z,), eps=1e-6, atol=1e-6, rtol=1e-4), name
