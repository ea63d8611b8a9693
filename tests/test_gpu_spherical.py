"""Spherical Bessel functions of real order n (spherical_bessel_{j,y,i,k}(n, z))
through the C ABI on the GPU: values and d/dz against mpmath (40 digits),
d/dn (central differences) and second derivatives within their difference
error, the reference's conventions for z < 0 and at the origin, parity with
the reference, float32 data, gradcheck."""

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden, run
from torchscience_b200 import special_functions as sf

pytestmark = pytest.mark.gpu

D = golden("spherical")
KINDS = "jyik"


def cuda(x, dtype=torch.float64):
    return torch.tensor(np.asarray(x), dtype=dtype, device="cuda")


def np_(t):
    return t.cpu().numpy().astype(np.float64)


def scales(kind, z, t):
    """(value, d/dz) error scales: relative for i and k; for j and y floored at
    1e-2 |z f'| (next to zeros) and 1e-3/|z| (the envelope's size)."""
    if kind in "ik":
        return np.abs(t[:, 0]), np.abs(t[:, 1])
    az = np.abs(z)
    s0 = np.maximum.reduce([np.abs(t[:, 0]), 1e-2 * az * np.abs(t[:, 1]), 1e-3 / az])
    s1 = np.maximum(np.abs(t[:, 1]), 1e-3 / az * (1 + 1 / az))
    return s0, s1


@pytest.mark.parametrize("kind", KINDS)
def test_values_and_derivatives(kind):
    name = f"spherical_bessel_{kind}"
    n, z, g, t = D[f"{name}_n"], D[f"{name}_z"], D[f"{name}_g"], D[f"{name}_truth"]
    (v,) = run(name, cuda(n), cuda(z))
    gn, gz = run(f"{name}_backward", cuda(g), cuda(n), cuda(z), n_out=2)
    v, gn, gz = np_(v), np_(gn), np_(gz)
    s0, s1 = scales(kind, z, t)
    m = np.isfinite(t).all(axis=1) & (s0 > 1e-290) & (np.abs(t[:, 0]) < 1e290) & (np.abs(t[:, 1]) < 1e290)
    e0 = np.abs(v - t[:, 0]) / s0
    e1 = np.abs(gz - g * t[:, 1]) / (np.abs(g) * s1)
    en = np.abs(gn - g * t[:, 2]) / (np.abs(g) * (np.abs(t[:, 2]) + np.abs(t[:, 0])))
    assert e0[m].max() <= 1e-13, f"value: {e0[m].max():.3e} at n={n[m][np.argmax(e0[m])]}, z={z[m][np.argmax(e0[m])]}"
    k1, kn = np.argmax(np.where(m, e1, 0)), np.argmax(np.where(m, en, 0))
    assert e1[m].max() <= 2e-12, f"d/dz: {e1[m].max():.3e} at n={n[k1]!r}, z={z[k1]!r}, got {gz[k1] / g[k1]!r}"
    # central differences in n: step error ~ h² ∂³f/∂n³, which grows like ln(z)³ f
    assert en[m].max() <= 1e-6, f"d/dn: {en[m].max():.3e} at n={n[kn]!r}, z={z[kn]!r}"


@pytest.mark.parametrize("kind", KINDS)
def test_second_derivatives(kind):
    name = f"spherical_bessel_{kind}"
    i = D[f"{name}_idx2"]
    n, z, t, t2 = D[f"{name}_n"][i], D[f"{name}_z"][i], D[f"{name}_truth"][i], D[f"{name}_truth2"]
    ggn, ggz, g = np.full_like(n, 0.5), np.full_like(n, -1.25), np.full_like(n, 2.0)
    o = [np_(x) for x in run(f"{name}_backward_backward", cuda(ggn), cuda(ggz), cuda(g), cuda(n), cuda(z), n_out=3)]
    fzz, fnz, fnn = t2[:, 0], t2[:, 1], t2[:, 2]
    want = [ggn * t[:, 2] + ggz * t[:, 1], g * (ggn * fnn + ggz * fnz), g * (ggn * fnz + ggz * fzz)]
    size = np.abs(t[:, 0]) + np.abs(t[:, 1]) + np.abs(t[:, 2]) + np.abs(fzz) + np.abs(fnz) + np.abs(fnn)
    m = np.isfinite(t2).all(axis=1) & np.isfinite(t).all(axis=1) & (size < 1e290) & (size > 1e-290)
    for q, tol in zip(range(3), (1e-8, 1e-6, 1e-7)):
        e = np.abs(o[q] - want[q]) / (4 * size)
        assert e[m].max() <= tol, f"output {q}: {e[m].max():.3e}"


@pytest.mark.parametrize("kind", KINDS)
def test_parity_with_reference(kind):
    """Where the reference is within 1e-10 of the truth, |ours - ref| <= 4 ulp +
    |ref - truth| + our tolerance; elsewhere ours is at least as close (the
    reference's real-order Bessel J is inaccurate for x > 20)."""
    name = f"spherical_bessel_{kind}"
    n, z, g, t = D[f"{name}_n"], D[f"{name}_z"], D[f"{name}_g"], D[f"{name}_truth"]
    (v,) = run(name, cuda(n), cuda(z))
    _, gz = run(f"{name}_backward", cuda(g), cuda(n), cuda(z), n_out=2)
    s0, s1 = scales(kind, z, t)
    for got, ref, want, sc, tol in ((np_(v), D[f"{name}_ref"], t[:, 0], s0, 1e-13),
                                    (np_(gz), D[f"{name}_ref_grad"][:, 1], g * t[:, 1], np.abs(g) * s1, 2e-12)):
        m = np.isfinite(want) & np.isfinite(ref) & (sc > 1e-290) & (np.abs(want) < 1e290)
        ours_e, ref_e = np.abs(got - want) / sc, np.abs(ref - want) / sc
        good = m & (ref_e <= 1e-10)
        bad = good & (np.abs(got - ref) > 4 * np.spacing(np.abs(ref)) + np.abs(ref - want) + tol * sc)
        assert not bad.any(), f"agreement: n={n[bad][:3]!r}, z={z[bad][:3]!r}"
        worse = m & ~good & (ours_e > ref_e + tol)
        assert not worse.any(), f"closer: n={n[worse][:3]!r}, z={z[worse][:3]!r}, ours {ours_e[worse][:3]!r}"


@pytest.mark.parametrize("kind", KINDS)
def test_reference_special_points(kind):
    """The origin (|z| < 1e-12), z < 0 with integer n, NaN: the reference's values
    and d/dz."""
    name = f"spherical_bessel_{kind}"
    sn, sz = D[f"{name}_special_n"], D[f"{name}_special_z"]
    (v,) = run(name, cuda(sn), cuda(sz))
    _, dz = run(f"{name}_backward", cuda(np.ones_like(sn)), cuda(sn), cuda(sz), n_out=2)
    assert np.allclose(np_(v), D[f"{name}_special_ref"], rtol=1e-12, atol=0, equal_nan=True)
    assert np.allclose(np_(dz), D[f"{name}_special_ref_grad"][:, 1], rtol=1e-10, atol=0, equal_nan=True)


@pytest.mark.parametrize("kind", KINDS)
def test_float32_data_is_the_fp64_value_rounded_once(kind):
    name = f"spherical_bessel_{kind}"
    n32, z32 = D[f"{name}_n"].astype(np.float32), D[f"{name}_z"].astype(np.float32)
    (v32,) = run(name, cuda(n32, torch.float32), cuda(z32, torch.float32))
    (v64,) = run(name, cuda(n32.astype(np.float64)), cuda(z32.astype(np.float64)))
    assert torch.equal(v32.isnan(), v64.float().isnan())
    fin = ~v32.isnan()
    assert torch.equal(v32[fin], v64.float()[fin])


def test_gradcheck():
    gen = torch.Generator(device="cuda").manual_seed(19)
    n = (torch.rand(5, device="cuda", dtype=torch.float64, generator=gen) * 3 + 0.2).requires_grad_()
    z = (torch.rand(5, device="cuda", dtype=torch.float64, generator=gen) * 6 + 0.5).requires_grad_()
    for kind in KINDS:
        fn = getattr(sf, f"spherical_bessel_{kind}")
        assert torch.autograd.gradcheck(fn, (n, z), eps=1e-6, atol=1e-6, rtol=1e-4), kind
