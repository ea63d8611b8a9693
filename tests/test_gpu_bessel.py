"""Bessel J, Y, I, K of real order and J_0 through the C ABI on the GPU: FP64
against scipy (AMOS) and mpmath, parity with the reference in its accurate
bands, mixed FP32 against FP64, ν-derivatives, reference conventions,
gradcheck, and the Wronskian identities at config-3 size."""

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden, rel_err, run

pytestmark = pytest.mark.gpu

D = golden("bessel")
NU, X, G = D["nu"], D["x"], D["g"]
OPS = {"j": "bessel_j", "y": "bessel_y", "i": "modified_bessel_i", "k": "modified_bessel_k"}


def cuda(a, dtype=torch.float64):
    return torch.tensor(np.asarray(a), dtype=dtype, device="cuda")


def fwd_and_dx(key, nu, x, dtype=torch.float64):
    n, z = cuda(nu, dtype), cuda(x, dtype)
    (v,) = run(OPS[key], n, z)
    g = torch.ones_like(z)
    _, dz = run(OPS[key] + "_backward", g, n, z, n_out=2)
    return v.cpu().numpy().astype(np.float64), dz.cpu().numpy().astype(np.float64)


def envelope(key):
    if key in "jy":
        return np.sqrt(D["truth_j"] ** 2 + D["truth_y"] ** 2), np.sqrt(D["truth_jp"] ** 2 + D["truth_yp"] ** 2)
    return np.abs(D[f"truth_{key}"]), np.abs(D[f"truth_{key}p"])


@pytest.mark.parametrize("key", list(OPS))
def test_fp64_values_and_x_derivatives_against_scipy(key):
    v, dv = fwd_and_dx(key, NU, X)
    tv, td = D[f"truth_{key}"], D[f"truth_{key}p"]
    ev, ed = envelope(key)
    fin = np.isfinite(tv) & (np.abs(tv) < 1e300) & (np.abs(tv) > 1e-300)
    # away from zeros: relative; near zeros: relative to the local envelope
    for got, tru, env in ((v, tv, ev), (dv, td, ed)):
        m = fin & np.isfinite(tru) & (np.abs(tru) > 1e-300) & (np.abs(tru) < 1e300)
        err = np.abs(got - tru) / np.maximum(np.abs(tru), 1e-3 * env)
        assert np.nanmax(err[m]) <= 5e-11, f"{key}: worst {np.nanmax(err[m]):.3e}"
        assert np.nanmedian(err[m]) <= 1e-14


def test_fp64_near_the_zeros_of_j0_and_j1():
    """Config-3 stress points within 1e-6 of the first 100 zeros of J0, J1 (mpmath truth)."""
    n, z = cuda(D["zero_nu"]), cuda(D["zero_x"])
    (v,) = run("bessel_j", n, z)
    e = rel_err(v.cpu().numpy(), D["zero_truth_j"])
    assert e.max() <= 1e-8, f"near-zero rel err {e.max():.3e}"
    (v0,) = run("bessel_j_0", cuda(D["zero_x"][:100]))
    e0 = rel_err(v0.cpu().numpy(), D["zero_truth_j"][:100])
    assert e0.max() <= 1e-8


@pytest.mark.parametrize("key", list(OPS))
def test_fp64_parity_with_reference_in_its_accurate_bands(key):
    """|ours - ref| <= 4 ulp + |ref - truth| + 5e-11 relative, where the reference
    is accurate: J, Y, I for x < 20, K for x < 1 (the reference-defect bands
    are graded against truth only)."""
    v, _ = fwd_and_dx(key, NU, X)
    ref, tru = D[f"ref_{key}"], D[f"truth_{key}"]
    band = X < (1.0 if key == "k" else 20.0)
    env, _ = envelope(key)
    m = band & np.isfinite(ref) & np.isfinite(tru) & (np.abs(tru) > 1e-300) & (np.abs(tru) < 1e300)
    allowed = 4 * np.spacing(np.abs(ref)) + np.abs(ref - tru) + 5e-11 * np.maximum(np.abs(tru), 1e-3 * env)
    assert np.all((np.abs(v - ref) <= allowed)[m])


@pytest.mark.parametrize("key", list(OPS))
def test_mixed_within_1e6_of_fp64(key):
    nu32, x32 = NU.astype(np.float32), X.astype(np.float32)
    vm, dm = fwd_and_dx(key, nu32, x32, torch.float32)
    vd, dd = fwd_and_dx(key, nu32.astype(np.float64), x32.astype(np.float64))
    normal = (np.abs(vd) > 1.2e-38) & (np.abs(vd) < 3e38)
    e = rel_err(vm, vd)
    assert e[normal].max() <= 1e-6, f"{key} mixed value {e[normal].max():.3e}"
    # derivative: J' has zeros inside x < 2 where FP32 cancels; judged against |C| there
    normal_d = (np.abs(dd) > 1.2e-38) & (np.abs(dd) < 3e38) & normal
    ed = np.abs(dm - dd) / np.maximum(np.abs(dd), 1e-2 * np.abs(vd) / np.maximum(x32, 1e-30))
    assert ed[normal_d].max() <= 1e-6, f"{key} mixed d/dx {ed[normal_d].max():.3e}"


@pytest.mark.parametrize("key", ["j", "k"])
def test_nu_derivative_against_mpmath(key):
    i = D["dnu_idx"]
    n, z = cuda(NU[i]), cuda(X[i])
    gn, _ = run(OPS[key] + "_backward", torch.ones_like(z), n, z, n_out=2)
    tru = D[f"truth_dnu_{key}"]
    env, _ = envelope(key)
    err = np.abs(gn.cpu().numpy() - tru) / np.maximum(np.abs(tru), 1e-3 * env[i] + 1e-300)
    m = np.isfinite(tru) & (np.abs(tru) < 1e300)
    assert np.median(err[m]) <= 1e-8 and err[m].max() <= 1e-5, f"{key} d/dnu {err[m].max():.3e}"


def test_reference_conventions():
    n = cuda([0.0, 1.0, -1.0, -0.5, 2.0, 1.5, 0.0, 3.0])
    z = cuda([0.0, 0.0, 0.0, 0.0, -1.0, -1.0, np.inf, -2.0])
    (j,) = run("bessel_j", n, z)
    j = j.cpu().numpy()
    assert j[0] == 1 and j[1] == 0 and j[2] == 0 and np.isinf(j[3])
    import scipy.special as sp

    assert j[4] == pytest.approx(sp.jv(2, 1.0), rel=1e-14)  # J_2(-1) = J_2(1)
    assert j[5] == pytest.approx(np.cos(1.5 * np.pi) * sp.jv(1.5, 1.0), abs=1e-15)
    assert j[6] == 0
    assert j[7] == pytest.approx(-sp.jv(3, 2.0), rel=1e-14)
    (y,) = run("bessel_y", cuda([0.5, 0.5, 0.5, 2.0]), cuda([0.0, -1.0, np.inf, 3.0]))
    y = y.cpu().numpy()
    assert y[0] == -np.inf and np.isnan(y[1]) and y[2] == 0 and y[3] == pytest.approx(sp.yv(2, 3.0), rel=1e-14)
    (k,) = run("modified_bessel_k", cuda([0.5, 0.5, -2.5, 2.5]), cuda([0.0, -1.0, 4.0, 4.0]))
    k = k.cpu().numpy()
    assert k[0] == np.inf and np.isnan(k[1]) and k[2] == k[3]
    (i,) = run("modified_bessel_i", cuda([0.0, 2.0, 3.0, -2.5]), cuda([0.0, -1.5, -1.5, 1.2]))
    i = i.cpu().numpy()
    assert i[0] == 1 and i[1] == pytest.approx(sp.iv(2, 1.5), rel=1e-14) and i[2] == pytest.approx(-sp.iv(3, 1.5), rel=1e-14)
    assert i[3] == pytest.approx(sp.iv(-2.5, 1.2), rel=1e-13)
    (j0,) = run("bessel_j_0", cuda([0.0, 2.404825557695773, -3.0]))
    assert j0.cpu().numpy()[0] == 1 and abs(j0.cpu().numpy()[1]) < 1e-15
    assert j0.cpu().numpy()[2] == pytest.approx(sp.j0(3.0), rel=1e-14)


def test_gradcheck_and_gradgradcheck():
    from torchscience_b200 import special_functions as sf

    gen = torch.Generator(device="cuda").manual_seed(3)
    n = (torch.rand(5, device="cuda", dtype=torch.float64, generator=gen) * 4 + 0.3).requires_grad_()
    z = (torch.rand(5, device="cuda", dtype=torch.float64, generator=gen) * 6 + 0.5).requires_grad_()
    for fn in (sf.bessel_j, sf.bessel_y, sf.modified_bessel_i, sf.modified_bessel_k):
        assert torch.autograd.gradcheck(fn, (n, z), eps=1e-6, atol=1e-6, rtol=1e-4)
        assert torch.autograd.gradgradcheck(fn, (n, z), eps=1e-5, atol=1e-4, rtol=1e-3)
    assert torch.autograd.gradcheck(sf.bessel_j_0, (z,), eps=1e-6, atol=1e-7)
    assert torch.autograd.gradgradcheck(sf.bessel_j_0, (z,), eps=1e-6, atol=1e-6)


def test_wronskians_at_config3_size():
    """J_ν Y'_ν - J'_ν Y_ν = 2/(πx) and I_ν K'_ν - I'_ν K_ν = -1/x over 2^24
    points with ν ~ U(0, 20), x ~ LogU(1e-3, 1e3) (relative to the product scale)."""
    gen = torch.Generator(device="cuda").manual_seed(0)
    N = 1 << 24
    nu = torch.rand(N, device="cuda", dtype=torch.float64, generator=gen) * 20
    x = torch.exp(torch.empty(N, device="cuda", dtype=torch.float64).uniform_(np.log(1e-3), np.log(1e3), generator=gen))
    ones = torch.ones_like(x)
    (j,) = run("bessel_j", nu, x)
    (y,) = run("bessel_y", nu, x)
    _, jp = run("bessel_j_backward", ones, nu, x, n_out=2)
    _, yp = run("bessel_y_backward", ones, nu, x, n_out=2)
    w = j * yp - jp * y
    scale = (j * yp).abs() + (jp * y).abs()
    ok = torch.isfinite(scale) & (scale < 1e300)
    r = ((w - 2 / (np.pi * x)).abs() / scale)[ok]
    assert r.max().item() <= 1e-10
    (i,) = run("modified_bessel_i", nu, x)
    (k,) = run("modified_bessel_k", nu, x)
    _, ip = run("modified_bessel_i_backward", ones, nu, x, n_out=2)
    _, kp = run("modified_bessel_k_backward", ones, nu, x, n_out=2)
    w = i * kp - ip * k
    scale = (i * kp).abs() + (ip * k).abs()
    ok = torch.isfinite(scale) & (scale < 1e300) & (scale > 1e-300)
    r = ((w + 1 / x).abs() / scale)[ok]
    assert r.max().item() <= 1e-10
