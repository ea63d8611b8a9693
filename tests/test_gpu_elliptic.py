"""Complete elliptic integrals K(m), E(m) through the C ABI on the GPU."""

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401
from tests._util import golden, rel_err, run

pytestmark = pytest.mark.gpu

D = golden("elliptic")
M, G = D["m"], D["g"]
NAMES = {"k": "complete_legendre_elliptic_integral_k", "e": "complete_legendre_elliptic_integral_e"}


def cuda(a, dtype=torch.float64):
    return torch.tensor(np.asarray(a), dtype=dtype, device="cuda")


@pytest.mark.parametrize("key", ["k", "e"])
def test_fp64_against_truth_and_reference(key):
    (y,) = run(NAMES[key], cuda(M))
    y = y.cpu().numpy()
    e = rel_err(y, D[f"truth_{key}"])
    assert e.max() <= 2e-15, f"{key}: {e.max():.3e}"
    inside = (M >= 0) & (M < 1 - 1e-12)
    ref, tru = D[f"ref_{key}"], D[f"truth_{key}"]
    allowed = 4 * np.spacing(np.abs(ref)) + np.abs(ref - tru) + 2e-15 * np.abs(tru)
    assert np.all((np.abs(y - ref) <= allowed)[inside])


@pytest.mark.parametrize("key", ["k", "e"])
def test_fp64_derivatives_against_truth(key):
    m, g = cuda(M), cuda(G)
    (gy,) = run(NAMES[key] + "_backward", g, m)
    e = rel_err(gy.cpu().numpy(), G * D[f"truth_d{key}"])
    assert e.max() <= 1e-13, f"d{key}/dm: {e.max():.3e}"
    gg = cuda(np.roll(G, 3))
    o0, o1 = run(NAMES[key] + "_backward_backward", gg, g, m, n_out=2)
    e2 = rel_err(o1.cpu().numpy(), np.roll(G, 3) * G * D[f"truth_d{key}{key}"])
    assert e2.max() <= 1e-11, f"d2{key}/dm2: {e2.max():.3e}"


@pytest.mark.parametrize("key", ["k", "e"])
def test_mixed_within_1e6_of_fp64(key):
    m32 = M.astype(np.float32)
    m32 = m32[m32 < 1]
    (ym,) = run(NAMES[key], cuda(m32, torch.float32))
    (yd,) = run(NAMES[key], cuda(m32.astype(np.float64)))
    e = rel_err(ym.cpu().numpy(), yd.cpu().numpy())
    assert e.max() <= 1e-6, f"mixed {key}: {e.max():.3e}"
    g32 = G[: m32.size].astype(np.float32)
    (gm,) = run(NAMES[key] + "_backward", cuda(g32, torch.float32), cuda(m32, torch.float32))
    (gd,) = run(NAMES[key] + "_backward", cuda(g32.astype(np.float64)), cuda(m32.astype(np.float64)))
    e = rel_err(gm.cpu().numpy(), gd.cpu().numpy())
    assert e.max() <= 1e-6, f"mixed d{key}: {e.max():.3e}"


def test_special_values():
    m = cuda([0.0, 1.0, 1.5, -np.inf, np.nan])
    (k,) = run(NAMES["k"], m)
    (e,) = run(NAMES["e"], m)
    k, e = k.cpu().numpy(), e.cpu().numpy()
    assert k[0] == pytest.approx(np.pi / 2, rel=1e-16) and e[0] == pytest.approx(np.pi / 2, rel=1e-16)
    assert np.isinf(k[1]) and e[1] == 1.0
    assert np.isnan(k[2]) and np.isnan(e[2]) and np.isnan(k[4])
    assert k[3] == 0.0 and np.isinf(e[3])


def test_legendre_relation_at_config5_size():
    """E(m)K(1-m) + E(1-m)K(m) - K(m)K(1-m) = π/2 over 2^26 points, m ~ U(0, 1-1e-9)."""
    from torchscience_b200 import special_functions as sf

    gen = torch.Generator(device="cuda").manual_seed(0)
    m = torch.rand(1 << 26, generator=gen, device="cuda", dtype=torch.float64) * (1 - 1e-9)
    m = m.clamp(1e-9, 1 - 1e-9)
    k, e = sf.complete_legendre_elliptic_integral_k(m), sf.complete_legendre_elliptic_integral_e(m)
    k1, e1 = sf.complete_legendre_elliptic_integral_k(1 - m), sf.complete_legendre_elliptic_integral_e(1 - m)
    r = e * k1 + e1 * k - k * k1 - np.pi / 2
    assert r.abs().max().item() <= 1e-13
