"""lnΓ, Γ, ψ, ψ' through the C ABI on the GPU: FP64 kernels against scipy/mpmath
truth and against the reference's own outputs; mixed FP32 kernels against the
FP64 kernels; first and second derivatives."""

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401  (loads the libraries)
from tests._util import golden, rel_err, run, ulp_err

pytestmark = pytest.mark.gpu

D = golden("gamma_family")
X, G = D["x"], D["g"]
GG = np.roll(G, 17)
ROOT_PSI = 1.4616321449683623

TRUTH = {
    "log_gamma": D["truth_log_gamma"],
    "gamma": D["truth_gamma"],
    "digamma": D["truth_digamma"],
    "trigamma": D["truth_polygamma1"],
}
D1 = {
    "log_gamma": D["truth_digamma"],
    "gamma": D["truth_gamma"] * D["truth_digamma"],
    "digamma": D["truth_polygamma1"],
    "trigamma": D["truth_polygamma2"],
}
D2 = {
    "log_gamma": D["truth_polygamma1"],
    "gamma": None,  # formed per test in overflow-safe order
    "digamma": D["truth_polygamma2"],
    "trigamma": D["truth_polygamma3"],
}


def cuda(a, dtype=torch.float64):
    return torch.tensor(np.asarray(a), dtype=dtype, device="cuda")


def band(name, x):
    """Cancellation bands: zeros of the function, where relative error is not meaningful."""
    if name == "log_gamma":
        return (np.abs(x - 1) < 0.1) | (np.abs(x - 2) < 0.1) | (x < 0)
    if name == "digamma":
        return (np.abs(x - ROOT_PSI) < 0.1) | (x < 0)
    return x < 0


# Error bounds of the FP64 kernels against truth outside the bands:
# |err| <= TOL64 * |value| + 2e-16 (an absolute floor for values near zeros).
TOL64 = {"log_gamma": 4e-15, "gamma": 1e-14, "digamma": 4e-15, "trigamma": 4e-15}


@pytest.mark.parametrize("name", list(TRUTH))
def test_fp64_forward_against_truth(name):
    (y,) = run(name, cuda(X))
    y = y.cpu().numpy()
    b = band(name, X)
    tru = TRUTH[name]
    over = np.abs(y - tru) / (TOL64[name] * np.abs(tru) + 2e-16)
    over = np.where(np.isinf(y) & np.isinf(tru), 0.0, over)
    assert over[~b].max() <= 1.0, f"{name}: worst error/bound {over[~b].max():.3f}"
    # inside the bands: absolute error relative to the function's local scale
    scale = np.maximum(1.0, np.abs(TRUTH[name]))
    ea = np.abs(y - TRUTH[name]) / scale
    assert np.nanmax(ea[b]) <= 1e-12, f"{name}: band abs err {np.nanmax(ea[b]):.3e}"


@pytest.mark.parametrize("name", list(TRUTH))
def test_fp64_forward_parity_with_reference(name):
    """Agreement with the reference's own outputs: |ours - ref| <= 4 ulp +
    |ref - truth| + our stated bound, in the reference-accurate band (x > 0,
    away from zeros; digamma/trigamma use a truncated 3-term asymptotic in
    the reference, a documented defect band, and are graded against truth)."""
    if name in ("digamma", "trigamma"):
        pytest.skip("reference digamma/trigamma are in their defect band (~1e-8 truncation)")
    (y,) = run(name, cuda(X))
    y = y.cpu().numpy()
    ref, tru = D[f"ref_{name}"], TRUTH[name]
    m = ~band(name, X) & (X < 170)
    allowed = 4 * np.spacing(np.abs(ref)) + np.abs(ref - tru) + TOL64[name] * np.abs(tru) + 2e-16
    assert np.all(np.abs(y - ref)[m] <= allowed[m])
    strict = np.mean((np.abs(y - ref) <= 4 * np.spacing(np.abs(ref)) + np.abs(ref - tru))[m])
    print(f"{name}: {100 * strict:.1f}% of points within 4 ulp of the reference + its own error")


@pytest.mark.parametrize("name", list(TRUTH))
def test_fp64_backward_and_double_backward(name):
    x, g, gg = cuda(X), cuda(G), cuda(GG)
    (gx,) = run(name + "_backward", g, x)
    e = rel_err(gx.cpu().numpy(), G * D1[name])
    b = band(name, X) | (np.abs(X - ROOT_PSI) < 0.1 if name in ("log_gamma", "gamma") else False)
    assert e[~b].max() <= 2e-14, f"{name} backward: {e[~b].max():.3e}"
    o0, o1 = run(name + "_backward_backward", gg, g, x, n_out=2)
    e0 = rel_err(o0.cpu().numpy(), GG * D1[name])
    if name == "gamma":  # scale before multiplying by Γ, as the kernel does, so the truth stays finite
        want1 = (GG * G * (D["truth_digamma"] ** 2 + D["truth_polygamma1"])) * D["truth_gamma"]
    else:
        want1 = GG * G * D2[name]
    e1 = rel_err(o1.cpu().numpy(), want1)
    assert e0[~b].max() <= 2e-14
    assert e1[~b].max() <= 2e-13, f"{name} double backward: {e1[~b].max():.3e}"


@pytest.mark.parametrize("name", list(TRUTH))
def test_mixed_forward_within_1e6_of_fp64(name):
    x32 = X.astype(np.float32)
    (ym,) = run(name, cuda(x32, torch.float32))
    (yd,) = run(name, cuda(x32.astype(np.float64)))
    ym = ym.cpu().numpy().astype(np.float64)
    yd = yd.cpu().numpy()
    yd_f32 = yd.astype(np.float32).astype(np.float64)  # overflow to inf where float32 does
    ok = np.isinf(yd_f32) & np.isinf(ym)
    e = np.where(ok, 0.0, rel_err(ym, yd))
    b = np.zeros_like(X, dtype=bool)
    if name == "log_gamma":  # zeros of lnΓ at 1 and 2: compare absolutely
        b = (np.abs(x32 - 1) < 0.1) | (np.abs(x32 - 2) < 0.1)
        assert np.abs(ym - yd)[b].max() <= 1e-7
    if name in ("log_gamma", "digamma"):  # zeros of lnΓ / ψ on the negative axis
        neg = x32 < 0
        assert (np.abs(ym - yd) / np.maximum(1, np.abs(yd)))[neg].max() <= 1e-6
        b |= neg
    assert e[~b].max() <= 1e-6, f"{name} mixed: {e[~b].max():.3e}"


@pytest.mark.parametrize("name", list(TRUTH))
def test_mixed_backward_within_1e6_of_fp64(name):
    x32 = X.astype(np.float32)
    g32 = G.astype(np.float32)
    (gm,) = run(name + "_backward", cuda(g32, torch.float32), cuda(x32, torch.float32))
    (gd,) = run(name + "_backward", cuda(g32.astype(np.float64)), cuda(x32.astype(np.float64)))
    gm, gd = gm.cpu().numpy().astype(np.float64), gd.cpu().numpy()
    fin = np.abs(gd) < 3e38
    b = (x32 < 0) | ~fin
    if name in ("log_gamma", "gamma"):
        b |= np.abs(x32 - ROOT_PSI) < 0.05
    e = rel_err(gm, gd)
    assert e[~b].max() <= 1e-6, f"{name} mixed backward: {e[~b].max():.3e}"


def test_full_size_properties():
    """Size-independent identities at config-1 size (2^20): lnΓ(x+1) = lnΓ(x) + ln x,
    ψ(x+1) = ψ(x) + 1/x, ψ'(x) - ψ'(x+1) = 1/x², Γ(x+1) = xΓ(x)."""
    gen = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand(1 << 20, generator=gen, device="cuda", dtype=torch.float64) * 49.99 + 0.01
    from torchscience_b200 import special_functions as sf

    lg = sf.log_gamma(x + 1) - sf.log_gamma(x) - torch.log(x)
    assert lg.abs().max().item() < 1e-12
    d = sf.digamma(x + 1) - sf.digamma(x) - 1 / x
    assert (d.abs() / (1 + sf.digamma(x).abs())).max().item() < 1e-13
    t = (sf.trigamma(x) - sf.trigamma(x + 1)) * x * x - 1
    assert t.abs().max().item() < 1e-12
    g = sf.gamma(x + 1) / (x * sf.gamma(x)) - 1
    assert g[x < 150].abs().max().item() < 1e-13
