"""Generates the committed golden fixtures under tests/golden/.

Run here, where the reference sources exist (the GPU box has only the
fixtures):

    python oracle/build_ref.py && python tests/golden/make_golden.py

Each fixture holds seeded inputs drawn from the distributions of the
benchmark configurations (small samples), the
reference's own outputs for them (oracle/_ref/libref_scalar.so, i.e. the
reference's scalar templates compiled from its sources) and high-accuracy
values from scipy 1.18 / mpmath 1.3 ("truth").
"""

from __future__ import annotations

import sys
from pathlib import Path

import mpmath as mp
import numpy as np
import scipy.special as sp

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent
mp.mp.dps = 40


def lu(rng, lo, hi, n):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n))


def ref(name, p, *ins):
    r = O.reference(name, p, *ins)
    if r is None:
        raise SystemExit("oracle/_ref/libref_scalar.so missing: run python oracle/build_ref.py first")
    return r


def gamma_family():
    rng = np.random.default_rng(0)
    x = np.concatenate(
        [
            rng.uniform(0.01, 50.0, 2048),  # config 1 distribution
            lu(rng, 0.1, 100.0, 1024),  # config 5 k distribution
            rng.uniform(-20.0, 0.0, 256),  # reflection region
            rng.uniform(1.3, 1.6, 128),  # around the digamma root
            np.array([0.5, 1.0, 2.0, 3.0, 4.0, 5.0, 10.0, 100.0, 171.0, 1e-3, 1e-8]),
        ]
    )
    g = rng.standard_normal(x.size)
    d = {"x": x, "g": g}
    for nm in ["log_gamma", "gamma", "digamma", "trigamma"]:
        d[f"ref_{nm}"] = ref(nm, 0, x)[0]
        d[f"ref_{nm}_backward"] = ref(nm, 1, g, x)[0]
    d["truth_log_gamma"] = sp.gammaln(x)
    d["truth_gamma"] = sp.gamma(x)
    d["truth_digamma"] = sp.psi(x)
    for k in (1, 2, 3):
        d[f"truth_polygamma{k}"] = sp.polygamma(k, x)
    # mpmath for the sign-carrying reflection region and the digamma root band
    d["truth_digamma"] = np.array([float(mp.digamma(mp.mpf(v))) if v <= 0 or 1.3 < v < 1.6 else sp.psi(v) for v in x])
    np.savez_compressed(OUT / "gamma_family.npz", **d)


def igamma():
    rng = np.random.default_rng(1)
    a_grid = lu(rng, 1e-2, 1e3, 48)
    x_grid = lu(rng, 1e-3, 2e3, 48)
    A, X = np.meshgrid(a_grid, x_grid, indexing="ij")
    a_s = lu(rng, 1e-2, 1e3, 1024)
    x_s = a_s * (1.0 + rng.uniform(-1e-2, 1e-2, a_s.size))  # |x - a| < 1e-2 a stress set
    a = np.concatenate([A.ravel(), a_s, [1.0, 1.0, 2.0, 0.5, 10.0]])
    x = np.concatenate([X.ravel(), x_s, [0.0, 100.0, 1e-300, 0.25, 9.5]])
    g = rng.standard_normal(a.size)
    d = {"a": a, "x": x, "g": g}
    for nm in ["regularized_gamma_p", "regularized_gamma_q"]:
        d[f"ref_{nm}"] = ref(nm, 0, a, x)[0]
        ga, gx = ref(nm, 1, g, a, x)
        d[f"ref_{nm}_grad_a"], d[f"ref_{nm}_grad_x"] = ga, gx
    # mpmath at 40 digits: scipy's gammainc is only good to ~1e-12 at large a.
    d["truth_p"] = np.array([float(mp.gammainc(mp.mpf(ai), 0, mp.mpf(xi), regularized=True)) if ai > 0 and xi > 0 else sp.gammainc(ai, xi) for ai, xi in zip(a, x)])
    d["truth_q"] = np.array([float(mp.gammainc(mp.mpf(ai), mp.mpf(xi), mp.inf, regularized=True)) if ai > 0 and xi > 0 else sp.gammaincc(ai, xi) for ai, xi in zip(a, x)])
    # Derivatives from mpmath at 40 digits on a subsample.
    idx = rng.choice(a.size - 5, 160, replace=False)
    d["deriv_idx"] = idx
    pa, px, paa, pax, pxx = [], [], [], [], []
    for i in idx:
        ai, xi = mp.mpf(a[i]), mp.mpf(x[i])

        def P(aa, xx):
            return mp.gammainc(aa, 0, xx, regularized=True)

        def Q(aa, xx):
            return mp.gammainc(aa, xx, mp.inf, regularized=True)

        # Differentiate whichever of P, Q is small: the other is 1 - tiny and a
        # numerical derivative of it would lose the digits that matter.
        upper = xi > ai
        f = (lambda t: -Q(t, xi)) if upper else (lambda t: P(t, xi))
        pa.append(float(mp.diff(f, ai)))
        px.append(float(mp.exp((ai - 1) * mp.log(xi) - xi - mp.loggamma(ai))))
        paa.append(float(mp.diff(f, ai, 2)))
        pax.append(float(mp.diff(lambda t: mp.exp((t - 1) * mp.log(xi) - xi - mp.loggamma(t)), ai)))
        pxx.append(float(px[-1] * ((ai - 1) / xi - 1)))
    d["truth_pa"], d["truth_px"] = np.array(pa), np.array(px)
    d["truth_paa"], d["truth_pax"], d["truth_pxx"] = np.array(paa), np.array(pax), np.array(pxx)
    np.savez_compressed(OUT / "igamma.npz", **d)


def elliptic():
    rng = np.random.default_rng(2)
    m = np.concatenate(
        [
            rng.uniform(0.0, 1.0 - 1e-9, 2048),  # config 5 distribution
            1.0 - lu(rng, 1e-12, 1e-2, 256),  # near the logarithmic singularity
            rng.uniform(-10.0, 0.0, 128),  # negative parameter
            lu(rng, 1e-12, 0.1, 128),  # small m (series band)
            np.array([0.0, 0.5, -1.0, 0.9]),
        ]
    )
    g = rng.standard_normal(m.size)
    d = {"m": m, "g": g}
    for nm, key in [("complete_legendre_elliptic_integral_k", "k"), ("complete_legendre_elliptic_integral_e", "e")]:
        d[f"ref_{key}"] = ref(nm, 0, m)[0]
        d[f"ref_{key}_backward"] = ref(nm, 1, g, m)[0]
    K = np.array([float(mp.ellipk(mp.mpf(v))) for v in m])
    E = np.array([float(mp.ellipe(mp.mpf(v))) for v in m])
    d["truth_k"], d["truth_e"] = K, E
    dk, de, dkk, dee = [], [], [], []
    for v in m:
        mv = mp.mpf(v)
        if mv == 0:
            dk.append(float(mp.pi / 8))
            de.append(float(-mp.pi / 8))
            dkk.append(float(9 * mp.pi / 64))
            dee.append(float(-3 * mp.pi / 64))
            continue
        k, e = mp.ellipk(mv), mp.ellipe(mv)
        kp = (e - (1 - mv) * k) / (2 * mv * (1 - mv))
        ep = (e - k) / (2 * mv)
        dk.append(float(kp))
        de.append(float(ep))
        dkk.append(float(mp.diff(mp.ellipk, mv, 2)))
        dee.append(float(mp.diff(mp.ellipe, mv, 2)))
    d["truth_dk"], d["truth_de"] = np.array(dk), np.array(de)
    d["truth_dkk"], d["truth_dee"] = np.array(dkk), np.array(dee)
    np.savez_compressed(OUT / "elliptic.npz", **d)


def bessel():
    rng = np.random.default_rng(3)
    n = 3000
    nu = np.concatenate([rng.uniform(0.0, 20.0, n), rng.uniform(-5.0, 0.0, 300), np.arange(0, 6, dtype=float)])
    x = np.concatenate([lu(rng, 1e-3, 1e3, n), lu(rng, 1e-2, 50.0, 300), np.full(6, 3.7)])
    d = {"nu": nu, "x": x, "g": rng.standard_normal(nu.size)}
    for nm, key in [("bessel_j", "j"), ("bessel_y", "y"), ("modified_bessel_i", "i"), ("modified_bessel_k", "k")]:
        d[f"ref_{key}"] = ref(nm, 0, nu, x)[0]
    d["truth_j"], d["truth_y"] = sp.jv(nu, x), sp.yv(nu, x)
    d["truth_i"], d["truth_k"] = sp.iv(nu, x), sp.kv(nu, x)
    d["truth_jp"], d["truth_yp"] = sp.jvp(nu, x), sp.yvp(nu, x)
    d["truth_ip"], d["truth_kp"] = sp.ivp(nu, x), sp.kvp(nu, x)
    # Near the first 100 zeros of J0 and J1 (config 3 stress set): mpmath truth.
    z0, z1 = sp.jn_zeros(0, 100), sp.jn_zeros(1, 100)
    zs = np.concatenate([z0, z1])
    zn = np.concatenate([np.zeros(100), np.ones(100)])
    zx = zs * (1.0 + rng.uniform(-1e-6, 1e-6, zs.size))
    d["zero_nu"], d["zero_x"] = zn, zx
    d["zero_truth_j"] = np.array([float(mp.besselj(mp.mpf(a), mp.mpf(b))) for a, b in zip(zn, zx)])
    d["zero_truth_jp"] = np.array([float(mp.besselj(mp.mpf(a), mp.mpf(b), derivative=1)) for a, b in zip(zn, zx)])
    # ∂/∂ν on a subsample (mpmath).
    idx = rng.choice(n, 120, replace=False)
    d["dnu_idx"] = idx
    d["truth_dnu_j"] = np.array([float(mp.diff(lambda t: mp.besselj(t, mp.mpf(x[i])), mp.mpf(nu[i]))) for i in idx])
    d["truth_dnu_k"] = np.array([float(mp.diff(lambda t: mp.besselk(t, mp.mpf(x[i])), mp.mpf(nu[i]))) for i in idx])
    np.savez_compressed(OUT / "bessel.npz", **d)


def bessel01():
    """J0 and J1 on the order-0/1 path: uniform and log-uniform arguments, both
    signs, and points within relative 1e-13..1e-3 of the zeros of J0 and J1
    below 60, with mpmath values of J0, J1 and J0'', and the reference's
    bessel_j_0 forward and backward."""
    rng = np.random.default_rng(8)
    z0, z1 = sp.jn_zeros(0, 19), sp.jn_zeros(1, 19)
    zs = np.concatenate([z0, z1])
    near = np.repeat(zs, 8) * (1.0 + rng.choice([-1.0, 1.0], zs.size * 8) * lu(rng, 1e-13, 1e-3, zs.size * 8))
    x = np.concatenate([rng.uniform(0.0, 60.0, 2000), -rng.uniform(0.0, 60.0, 300), lu(rng, 1e-8, 1e6, 600), near])
    d = {"x": x, "g": rng.standard_normal(x.size)}
    d["truth_j0"] = np.array([float(mp.besselj(0, mp.mpf(v))) for v in x])
    d["truth_j1"] = np.array([float(mp.besselj(1, mp.mpf(v))) for v in x])
    d["truth_j0pp"] = np.array([float(mp.besselj(0, mp.mpf(v), derivative=2)) for v in x])
    d["ref_j0"] = ref("bessel_j_0", 0, x)[0]
    d["ref_j0_grad"] = ref("bessel_j_0", 1, d["g"], x)[0]
    np.savez_compressed(OUT / "bessel01.npz", **d)


def hyp2f1():
    """2F1 fixtures: the reference's known answers, its scipy grid, a seeded
    sample of the benchmark distribution (a, b, c ~ U(-10, 10), c rejected
    within 1e-3 of a non-positive integer, z ~ U(-5, 0.9) w.p. 0.9 else
    U(0.9, 0.999)) with mpmath values, gradients and input condition numbers
    κ = Σ|x_i ∂F/∂x_i| / |F|, Hessians on a subsample, and the reference's
    outputs on its special points."""
    rng = np.random.default_rng(4)
    d = {}
    # Known answers, test__hypergeometric_2_f_1.py:2604-2703.
    kat = [(1.5, 2.5, 3.5, 0.3, 1.452767637957694), (-2.0, 3.0, 4.0, 0.7, 0.244), (1.0, 2.0, -1.0, 0.3, np.inf),
           (2.0, 3.0, 3.0, 0.3, 0.7 ** -2.0), (1.0, 2.0, 4.0, 0.9, 2.1789423102929675),
           (1.0, 2.0, 3.0, -5.0, 0.2566592424617554), (1.5, 2.5, 3.5, -2.0, 0.28453773594866716)]
    d["kat"] = np.array(kat)
    # The scipy grid of test__hypergeometric_2_f_1.py:327-345 and the z -> 1 sweep of :1944-1970.
    g = np.array([(a, b, c, z) for z in (0.1, 0.3, 0.5, 0.7) for a in (0.5, 1.0, 2.0) for b in (0.5, 1.0, 2.0)
                  for c in (1.0, 2.0, 3.0)] + [(0.3, 0.4, 2.0, z) for z in (0.99, 0.999, 0.9999, 0.99999)])
    d["grid"] = g
    d["grid_truth"] = np.array([float(mp.hyp2f1(*map(mp.mpf, r))) for r in g])
    # Integer c - a - b near z = 1 and z -> -inf (the degenerate connection formula).
    deg = np.array([(1.0, 2.0, 4.0, 0.999), (1.0, 2.0, 4.0, 0.9999), (1.0, 2.0, 3.0, 0.9995), (0.5, 1.5, 3.0, 0.9999),
                    (2.5, 1.5, 5.0, 0.99999), (1.0, 2.0, 3.0, -500.0), (1.5, 1.5, 2.0, -300.0)])
    d["degenerate"] = deg
    d["degenerate_truth"] = np.array([float(mp.hyp2f1(*map(mp.mpf, r))) for r in deg])
    # Benchmark-distribution sample.
    n = 1500
    a = rng.uniform(-10, 10, n)
    b = rng.uniform(-10, 10, n)
    c = rng.uniform(-10, 10, n)
    bad = (c <= 0) & (np.abs(c - np.round(c)) < 1e-3)
    while bad.any():
        c[bad] = rng.uniform(-10, 10, bad.sum())
        bad = (c <= 0) & (np.abs(c - np.round(c)) < 1e-3)
    z = np.where(rng.random(n) < 0.9, rng.uniform(-5, 0.9, n), rng.uniform(0.9, 0.999, n))
    d["a"], d["b"], d["c"], d["z"] = a, b, c, z
    d["ref"] = ref("hypergeometric_2_f_1", 0, a, b, c, z)[0]
    f = lambda A, B, C, Z: mp.hyp2f1(A, B, C, Z)  # noqa: E731
    truth, grad, kappa = np.empty(n), np.empty((n, 4)), np.empty(n)
    for i in range(n):
        X = [mp.mpf(v) for v in (a[i], b[i], c[i], z[i])]
        F = f(*X)
        gi = [mp.diff(f, X, tuple(int(j == k) for j in range(4))) for k in range(4)]
        truth[i] = float(F)
        grad[i] = [float(v) for v in gi]
        kappa[i] = float(sum(abs(X[k] * gi[k]) for k in range(4)) / abs(F))
    d["truth"], d["truth_grad"], d["kappa"] = truth, grad, kappa
    m = 300
    d["g"] = rng.standard_normal(m)
    d["ref_grad"] = np.stack(ref("hypergeometric_2_f_1", 1, d["g"], a[:m], b[:m], c[:m], z[:m]), axis=1)
    # Hessians [aa, ab, ac, az, bb, bc, bz, cc, cz, zz] on the first 60 points.
    pairs = [(0, 0), (0, 1), (0, 2), (0, 3), (1, 1), (1, 2), (1, 3), (2, 2), (2, 3), (3, 3)]
    hess = np.empty((60, 10))
    for i in range(60):
        X = [mp.mpf(v) for v in (a[i], b[i], c[i], z[i])]
        hess[i] = [float(mp.diff(f, X, tuple(int(p == j) + int(q == j) for j in range(4)))) for p, q in pairs]
    d["truth_hess"] = hess
    # Special points: the reference's early returns and their neighbourhoods.
    sp_pts = [(0.0, 2.0, 3.0, 0.4), (1.5, 0.0, 3.0, -2.0), (1.5, 2.5, 3.5, 0.0), (2.0, 1.5, 1.5, -0.7),
              (1.5, 2.0, 1.5, 0.6), (-3.0, 2.5, 4.5, 0.8), (2.5, -4.0, 1.5, -3.0), (-1.0, 2.0, -2.0, 0.5),
              (-3.0, 2.0, -2.0, 0.5), (1.0, 2.0, -3.0, 0.5), (0.5, 0.25, 2.0, 1.0), (1.5, 2.5, 3.0, 1.0),
              (2.0, 3.0, 3.5, -1.0), (0.5, 0.5, 3.0, -1.0), (1.0, 2.0, 3.0, 1.5), (1.0, 2.0, 3.0, np.nan),
              (np.nan, 2.0, 3.0, 0.5), (1.0, 2.0, 3.0, -1e-16), (1.2, 2.3, 3.4, 0.5), (1.2, 2.3, 3.4, -1.0 - 1e-12)]
    sp_pts = np.array(sp_pts)
    d["special"] = sp_pts
    d["special_ref"] = ref("hypergeometric_2_f_1", 0, *sp_pts.T)[0]
    np.savez_compressed(OUT / "hyp2f1.npz", **d)


def _dP_da(a, x):
    """∂P/∂a by mpmath, as -∂Q/∂a where x > a (P is then close to 1 and its
    difference quotient would lose the digits)."""
    a, x = mp.mpf(a), mp.mpf(x)
    if x > a:
        return -float(mp.diff(lambda t: mp.gammainc(t, x, mp.inf, regularized=True), a))
    return float(mp.diff(lambda t: mp.gammainc(t, 0, x, regularized=True), a))


def probability():
    """Gamma / chi-squared / Poisson CDF fixtures: seeded inputs, scipy values
    and densities, mpmath a-derivatives on a subsample, the reference's outputs
    and backward outputs, and its boundary cases (x <= 0, k < 0, NaN)."""
    import scipy.stats as st

    rng = np.random.default_rng(5)
    n = 3000
    d = {}
    # gamma
    x, sh, sc = lu(rng, 1e-3, 1e3, n), lu(rng, 0.1, 100.0, n), lu(rng, 0.1, 10.0, n)
    x[:20] = [0.0, -1.0, np.nan] + [1.0] * 17
    g = rng.standard_normal(n)
    d["gamma_x"], d["gamma_shape"], d["gamma_scale"], d["gamma_g"] = x, sh, sc, g
    with np.errstate(invalid="ignore"):
        d["gamma_truth"] = np.where(x > 0, st.gamma.cdf(x, sh, scale=sc), np.where(np.isnan(x), np.nan, 0.0))
        d["gamma_truth_pdf"] = np.where(x > 0, st.gamma.pdf(x, sh, scale=sc), np.where(np.isnan(x), np.nan, 0.0))
    d["gamma_ref"] = ref("gamma_cumulative_distribution", 0, x, sh, sc)[0]
    d["gamma_ref_grad"] = np.stack(ref("gamma_cumulative_distribution", 1, g, x, sh, sc), axis=1)
    idx = np.arange(20, 220)
    d["gamma_dshape_idx"] = idx
    d["gamma_truth_dshape"] = np.array([_dP_da(sh[i], mp.mpf(x[i]) / mp.mpf(sc[i])) for i in idx])
    # chi2
    x2, df = lu(rng, 1e-3, 1e3, n), lu(rng, 0.2, 200.0, n)
    x2[:3] = [0.0, -2.0, np.nan]
    g2 = rng.standard_normal(n)
    d["chi2_x"], d["chi2_df"], d["chi2_g"] = x2, df, g2
    with np.errstate(invalid="ignore"):
        d["chi2_truth"] = np.where(x2 > 0, st.chi2.cdf(x2, df), np.where(np.isnan(x2), np.nan, 0.0))
        d["chi2_truth_pdf"] = np.where(x2 > 0, st.chi2.pdf(x2, df), np.where(np.isnan(x2), np.nan, 0.0))
    d["chi2_ref"] = ref("chi2_cumulative_distribution", 0, x2, df)[0]
    d["chi2_ref_grad"] = np.stack(ref("chi2_cumulative_distribution", 1, g2, x2, df), axis=1)
    idx2 = np.arange(3, 203)
    d["chi2_ddf_idx"] = idx2
    d["chi2_truth_ddf"] = np.array([0.5 * _dP_da(df[i] / 2, mp.mpf(x2[i]) / 2) for i in idx2])
    # poisson
    k = np.concatenate([rng.integers(0, 120, n - 6).astype(float) + np.where(rng.random(n - 6) < 0.2, 0.5, 0.0),
                        [-1.0, -0.5, 0.0, 3.7, np.nan, 10.0]])
    rate = np.concatenate([lu(rng, 1e-2, 100.0, n - 6), [1.0, 1.0, 2.5, 2.5, 1.0, np.nan]])
    g3 = rng.standard_normal(n)
    d["poisson_k"], d["poisson_rate"], d["poisson_g"] = k, rate, g3
    kf = np.floor(k)
    with np.errstate(invalid="ignore"):
        d["poisson_truth"] = np.where(kf >= 0, st.poisson.cdf(kf, rate), np.where(np.isnan(kf), np.nan, 0.0))
        d["poisson_truth_drate"] = np.where(kf >= 0, -st.poisson.pmf(kf, rate), np.where(np.isnan(kf), np.nan, 0.0))
    d["poisson_ref"] = ref("poisson_cumulative_distribution", 0, k, rate)[0]
    d["poisson_ref_grad"] = np.stack(ref("poisson_cumulative_distribution", 1, g3, k, rate), axis=1)
    np.savez_compressed(OUT / "probability.npz", **d)


def probability_density():
    """Gamma and chi-squared densities with their gradients, and the chi-squared
    survival function: seeded inputs from the CDF fixtures' distributions,
    mpmath values (40 digits) of the density, its derivatives in x, shape
    (df) and scale, and of Q and its df-derivative on a subsample; the
    reference's outputs and backward outputs; boundary cases (x <= 0, NaN,
    the χ² density at x = 0 for df below, at and above 2)."""
    rng = np.random.default_rng(9)
    n = 2000
    d = {}

    def gpdf(x, a, s):
        x, a, s = mp.mpf(x), mp.mpf(a), mp.mpf(s)
        return mp.exp((a - 1) * mp.log(x) - x / s - a * mp.log(s) - mp.loggamma(a))

    # gamma density
    x, sh, sc = lu(rng, 1e-3, 1e3, n), lu(rng, 0.1, 100.0, n), lu(rng, 0.1, 10.0, n)
    x[:3] = [0.0, -1.0, np.nan]
    g = rng.standard_normal(n)
    d["gamma_x"], d["gamma_shape"], d["gamma_scale"], d["gamma_g"] = x, sh, sc, g
    t = np.zeros((n, 4))
    for i in range(n):
        if not x[i] > 0:
            t[i] = [np.nan if np.isnan(x[i]) else 0.0] + [0.0] * 3
            continue
        f = gpdf(x[i], sh[i], sc[i])
        X, a, s = mp.mpf(x[i]), mp.mpf(sh[i]), mp.mpf(sc[i])
        t[i] = [float(f), float(f * ((a - 1) / X - 1 / s)), float(f * (mp.log(X / s) - mp.digamma(a))),
                float(f * (X / s**2 - a / s))]
    d["gamma_truth"], d["gamma_truth_grad"] = t[:, 0], t[:, 1:]
    d["gamma_ref"] = ref("gamma_probability_density", 0, x, sh, sc)[0]
    d["gamma_ref_grad"] = np.stack(ref("gamma_probability_density", 1, g, x, sh, sc), axis=1)
    # chi-squared density
    x2, df = lu(rng, 1e-3, 1e3, n), lu(rng, 0.2, 200.0, n)
    x2[:6] = [0.0, 0.0, 0.0, -2.0, np.nan, 1.0]
    df[:6] = [1.0, 2.0, 3.0, 4.0, 4.0, np.nan]
    g2 = rng.standard_normal(n)
    d["chi2_x"], d["chi2_df"], d["chi2_g"] = x2, df, g2
    t2 = np.zeros((n, 3))
    for i in range(n):
        if np.isnan(x2[i]) or np.isnan(df[i]):
            t2[i] = [np.nan, 0.0, 0.0]
            continue
        if x2[i] <= 0:
            v = 0.0 if x2[i] < 0 else (np.inf if df[i] < 2 else (0.5 if df[i] == 2 else 0.0))
            t2[i] = [v, 0.0, 0.0]
            continue
        k, X = mp.mpf(df[i]) / 2, mp.mpf(x2[i])
        f = gpdf(X, k, 2)
        t2[i] = [float(f), float(f * ((k - 1) / X - mp.mpf(1) / 2)), float(f * (mp.log(X / 2) - mp.digamma(k)) / 2)]
    d["chi2_truth"], d["chi2_truth_grad"] = t2[:, 0], t2[:, 1:]
    d["chi2_ref"] = ref("chi2_probability_density", 0, x2, df)[0]
    d["chi2_ref_grad"] = np.stack(ref("chi2_probability_density", 1, g2, x2, df), axis=1)
    # chi-squared survival: Q(df/2, x/2)
    x3, df3 = lu(rng, 1e-3, 2e3, n), lu(rng, 0.2, 200.0, n)
    x3[:3] = [0.0, -1.0, np.nan]
    g3 = rng.standard_normal(n)
    d["sf_x"], d["sf_df"], d["sf_g"] = x3, df3, g3
    q = np.zeros(n)
    for i in range(n):
        if np.isnan(x3[i]):
            q[i] = np.nan
        elif x3[i] <= 0:
            q[i] = 1.0
        else:
            q[i] = float(mp.gammainc(mp.mpf(df3[i]) / 2, mp.mpf(x3[i]) / 2, mp.inf, regularized=True))
    d["sf_truth"] = q
    with np.errstate(invalid="ignore"):
        d["sf_truth_dx"] = np.array([0.0 if not v > 0 else -float(gpdf(v, mp.mpf(k) / 2, 2)) for v, k in zip(x3, df3)])
    idx = np.arange(3, 203)
    d["sf_ddf_idx"] = idx
    d["sf_truth_ddf"] = np.array([-0.5 * _dP_da(df3[i] / 2, mp.mpf(x3[i]) / 2) for i in idx])
    d["sf_ref"] = ref("chi2_survival", 0, x3, df3)[0]
    d["sf_ref_grad"] = np.stack(ref("chi2_survival", 1, g3, x3, df3), axis=1)
    np.savez_compressed(OUT / "probability_density.npz", **d)


def beta_family():
    """log_beta, beta and polygamma: seeded positive arguments over [1e-3, 1e6]
    (with a block of b << a, where ψ(a) - ψ(a+b) cancels), negative
    non-integer a, the reference's special points, and orders 0..30 of ψ^(n)
    at positive and negative z; mpmath values (40 digits) of ln|B|, B, the
    ψ and ψ' differences, ψ^(n), ψ^(n+1), ψ^(n+2); the reference's outputs."""
    rng = np.random.default_rng(10)
    n = 2000
    a = np.concatenate([lu(rng, 1e-3, 1e6, n), rng.uniform(0.05, 20.0, 400), -rng.uniform(0.0, 10.0, 200) - 1e-3])
    b = np.concatenate([lu(rng, 1e-3, 1e6, n), rng.uniform(0.05, 20.0, 400), rng.uniform(0.1, 10.0, 200)])
    b[:300] = a[:300] * lu(rng, 1e-12, 1e-3, 300)
    sa = np.array([0.0, -1.0, 1.0, 0.5, 2.0, np.nan, 1.0, np.inf, 3.0])
    sb = np.array([1.0, 1.0, 1.0, 0.5, 3.0, 1.0, np.nan, 2.0, 1e-300])
    d = {"a": a, "b": b, "special_a": sa, "special_b": sb, "g": rng.standard_normal(a.size)}
    cols = {k: [] for k in ("lnb", "b", "da", "db", "daa", "dbb", "dab")}
    for x, y in zip(a, b):
        X, Y = mp.mpf(x), mp.mpf(y)
        B = mp.gamma(X) * mp.gamma(Y) / mp.gamma(X + Y) if x < 0 else mp.beta(X, Y)
        cols["lnb"].append(float(mp.log(abs(B))))
        cols["b"].append(float(B))
        cols["da"].append(float(mp.digamma(X) - mp.digamma(X + Y)))
        cols["db"].append(float(mp.digamma(Y) - mp.digamma(X + Y)))
        cols["daa"].append(float(mp.psi(1, X) - mp.psi(1, X + Y)))
        cols["dbb"].append(float(mp.psi(1, Y) - mp.psi(1, X + Y)))
        cols["dab"].append(float(-mp.psi(1, X + Y)))
    for k, v in cols.items():
        d[f"truth_{k}"] = np.array(v)
    gg = rng.standard_normal((2, a.size))
    d["gg"] = gg
    for nm in ("log_beta", "beta"):
        d[f"ref_{nm}"] = ref(nm, 0, a, b)[0]
        d[f"ref_{nm}_grad"] = np.stack(ref(nm, 1, d["g"], a, b), axis=1)
        d[f"ref_{nm}_bb"] = np.stack(ref(nm, 2, gg[0], gg[1], d["g"], a, b), axis=1)
        d[f"ref_{nm}_special"] = ref(nm, 0, sa, sb)[0]
    # polygamma
    m = 1500
    pn = np.concatenate([rng.integers(0, 31, m).astype(float), [2.7, -0.5, -1.0, 4.0, 5.0, 4.0, 1.0, 2.0, 6.0]])
    pz = np.concatenate([lu(rng, 1e-3, 1e3, m - 300), -rng.uniform(0.0, 30.0, 300) - 1e-3,
                         [2.0, 2.0, 2.0, 0.0, -3.0, 2.0, 1.0, 0.5, -0.5]])
    d["pg_n"], d["pg_z"] = pn, pz
    t0, t1, t2 = [], [], []
    for k, z in zip(pn, pz):
        order = int(k) if k > -1 else -1
        Z = mp.mpf(z)
        pole = z <= 0 and z == int(z)
        for lst, o in ((t0, order), (t1, int(k + 1) if k + 1 > -1 else -1), (t2, int(k + 2) if k + 2 > -1 else -1)):
            lst.append(np.nan if o < 0 or pole else float(mp.polygamma(o, Z)))
    d["pg_truth"], d["pg_truth_d1"], d["pg_truth_d2"] = np.array(t0), np.array(t1), np.array(t2)
    d["pg_g"] = rng.standard_normal(pn.size)
    d["pg_ref"] = ref("polygamma", 0, pn, pz)[0]
    d["pg_ref_grad"] = np.stack(ref("polygamma", 1, d["pg_g"], pn, pz), axis=1)
    np.savez_compressed(OUT / "beta_family.npz", **d)


BESSEL_INT = {  # name: (mpmath function, order, domain sign: 1 = z > 0 only, 0 = both signs)
    "bessel_j_1": (mp.besselj, 1, 0), "bessel_y_0": (mp.bessely, 0, 1), "bessel_y_1": (mp.bessely, 1, 1),
    "modified_bessel_i_0": (mp.besseli, 0, 0), "modified_bessel_i_1": (mp.besseli, 1, 0),
    "modified_bessel_k_0": (mp.besselk, 0, 1), "modified_bessel_k_1": (mp.besselk, 1, 1)}


def bessel_int():
    """Integer orders 0 and 1 as unary ops: z log-uniform over [1e-6, 1e3] (to
    700 for I), z in [0, 60], negative z for the odd/even functions, points
    within relative 1e-10..1e-4 of the first zeros of J1, Y0, Y1; mpmath values
    (40 digits) of f, f', f''; the reference's forward, backward and double
    backward outputs; the reference's special points."""
    rng = np.random.default_rng(11)
    d = {}
    for name, (fn, order, pos_only) in BESSEL_INT.items():
        hi = 700.0 if name.startswith("modified_bessel_i") else 1e3
        z = np.concatenate([lu(rng, 1e-6, hi, 800), rng.uniform(0.0, 60.0, 400)])
        if not pos_only:
            z = np.concatenate([z, -lu(rng, 1e-6, 60.0, 200)])
        if name in ("bessel_j_1", "bessel_y_0", "bessel_y_1"):
            kind = {"bessel_j_1": (mp.besseljzero, 1), "bessel_y_0": (mp.besselyzero, 0), "bessel_y_1": (mp.besselyzero, 1)}[name]
            zs = np.array([float(kind[0](kind[1], k)) for k in range(1, 16)])
            z = np.concatenate([z, np.repeat(zs, 6) * (1 + rng.choice([-1.0, 1.0], 90) * lu(rng, 1e-10, 1e-4, 90))])
        g, gg = rng.standard_normal(z.size), rng.standard_normal(z.size)
        if name.startswith("modified_bessel_k"):  # mpmath's besselk takes no derivative order: closed forms
            def kd(v, n=order):
                v = mp.mpf(v)
                k0, k1 = mp.besselk(0, v), mp.besselk(1, v)
                if n == 0:
                    return [k0, -k1, k0 + k1 / v]
                return [k1, -k0 - k1 / v, k1 + k0 / v + 2 * k1 / v**2]

            t = np.array([[float(x) for x in kd(v)] for v in z])
        else:  # mpmath's derivative formulas return an mpc (zero imaginary part) for some z < 0
            t = np.array([[float(mp.re(fn(order, mp.mpf(v), derivative=k))) for k in range(3)] for v in z])
        d[f"{name}_z"], d[f"{name}_g"], d[f"{name}_gg"] = z, g, gg
        d[f"{name}_truth"] = t
        d[f"{name}_ref"] = ref(name, 0, z)[0]
        d[f"{name}_ref_grad"] = ref(name, 1, g, z)[0]
        d[f"{name}_ref_bb"] = np.stack(ref(name, 2, gg, g, z), axis=1)
        sz = np.array([0.0, -0.0, -1.0, np.inf, -np.inf, np.nan, 1e-13])
        d[f"{name}_special_z"] = sz
        d[f"{name}_special_ref"] = ref(name, 0, sz)[0]
        d[f"{name}_special_ref_grad"] = ref(name, 1, np.ones_like(sz), sz)[0]
    np.savez_compressed(OUT / "bessel_int.npz", **d)


SPH01 = {  # closed forms at 50 digits
    "spherical_bessel_j_0": lambda z: mp.sin(z) / z, "spherical_bessel_j_1": lambda z: mp.sin(z) / z**2 - mp.cos(z) / z,
    "spherical_bessel_y_0": lambda z: -mp.cos(z) / z,
    "spherical_bessel_y_1": lambda z: -mp.cos(z) / z**2 - mp.sin(z) / z,
    "spherical_bessel_i_0": lambda z: mp.sinh(z) / z,
    "spherical_bessel_i_1": lambda z: mp.cosh(z) / z - mp.sinh(z) / z**2,
    "spherical_bessel_k_0": lambda z: mp.pi / 2 * mp.exp(-z) / z,
    "spherical_bessel_k_1": lambda z: mp.pi / 2 * (1 + z) * mp.exp(-z) / z**2}


def spherical01():
    """Spherical Bessel functions of order 0 and 1: z uniform in [-30, 30],
    log-uniform magnitudes in [1e-8, 600] of both signs (k: [1e-8, 600]),
    points within relative 1e-10..1e-4 of the first zeros of j0, j1, y0, y1;
    values, first and second derivatives from the closed forms at 50 digits
    (mpmath); the reference's forward, backward and double backward outputs;
    the reference's special points."""
    mp.mp.dps = 50
    rng = np.random.default_rng(12)
    d = {}
    for name, f in SPH01.items():
        z = np.concatenate([rng.uniform(-30.0, 30.0, 500), lu(rng, 1e-8, 600.0, 500) * rng.choice([-1.0, 1.0], 500)])
        if name.startswith("spherical_bessel_k"):
            z = np.abs(z)
        if name in ("spherical_bessel_j_0", "spherical_bessel_j_1", "spherical_bessel_y_0", "spherical_bessel_y_1"):
            g0 = {"j_0": lambda k: k * mp.pi, "j_1": lambda k: mp.besseljzero(1.5, k),
                  "y_0": lambda k: (k - 0.5) * mp.pi, "y_1": lambda k: mp.besselyzero(1.5, k)}
            zr = np.array([float(g0[name[-3:]](k)) for k in range(1, 11)])
            z = np.concatenate([z, np.repeat(zr, 6) * (1 + rng.choice([-1.0, 1.0], 60) * lu(rng, 1e-10, 1e-4, 60))])
        g, gg = rng.standard_normal(z.size), rng.standard_normal(z.size)
        t = np.array([[float(mp.diff(f, mp.mpf(v), k)) if k else float(f(mp.mpf(v))) for k in range(3)] for v in z])
        d[f"{name}_z"], d[f"{name}_g"], d[f"{name}_gg"], d[f"{name}_truth"] = z, g, gg, t
        d[f"{name}_ref"] = ref(name, 0, z)[0]
        d[f"{name}_ref_grad"] = ref(name, 1, g, z)[0]
        d[f"{name}_ref_bb"] = np.stack(ref(name, 2, gg, g, z), axis=1)
        sz = np.array([0.0, -0.0, 1e-13, -1e-13, -1.0, np.inf, -np.inf, np.nan])
        d[f"{name}_special_z"] = sz
        d[f"{name}_special_ref"] = ref(name, 0, sz)[0]
        d[f"{name}_special_ref_grad"] = ref(name, 1, np.ones_like(sz), sz)[0]
    mp.mp.dps = 40
    np.savez_compressed(OUT / "spherical01.npz", **d)


def _sph_truth(kind, n, z):
    """The reference's convention of the spherical Bessel function of real order
    at 40 digits: sqrt(pi/(2|z|)) C_{n+1/2}(|z|) times, for z < 0, the factor
    (-1)^n or cos(pi n) (y: n + 1)."""
    fn = {"j": mp.besselj, "y": mp.bessely, "i": mp.besseli, "k": mp.besselk}[kind]
    az = abs(z)
    v = mp.sqrt(mp.pi / (2 * az)) * fn(n + mp.mpf(1) / 2, az)
    if z < 0:
        m = n + 1 if kind == "y" else n
        v *= mp.cos(mp.pi * m)
    return mp.re(v)


def spherical():
    """Spherical Bessel functions of real order n: n in {0..10} and U(-2.5, 10),
    z in U(0.05, 40) and LogU(1e-6, 300), negative z for j, y, i; mpmath values,
    d/dz and d/dn (40 digits), second derivatives on a subsample; the
    reference's forward and backward outputs and its special points."""
    rng = np.random.default_rng(13)
    d = {}
    for kind in "jyik":
        name = f"spherical_bessel_{kind}"
        m = 400
        n = np.where(rng.random(m) < 0.5, rng.integers(0, 11, m).astype(float), rng.uniform(-2.5, 10.0, m))
        z = np.where(rng.random(m) < 0.5, rng.uniform(0.05, 40.0, m), lu(rng, 1e-6, 300.0, m))
        if kind != "k":
            z = z * np.where(rng.random(m) < 0.2, -1.0, 1.0)
        g = rng.standard_normal(m)
        t = []
        for a, b in zip(n, z):
            A, Bz = mp.mpf(a), mp.mpf(b)
            t.append([float(_sph_truth(kind, A, Bz)), float(mp.diff(lambda u: _sph_truth(kind, A, u), Bz)),
                      float(mp.diff(lambda u: _sph_truth(kind, u, Bz), A))])
        d[f"{name}_n"], d[f"{name}_z"], d[f"{name}_g"] = n, z, g
        d[f"{name}_truth"] = np.array(t)
        idx = np.arange(0, m, 4)
        t2 = []
        for i in idx:
            A, Bz = mp.mpf(n[i]), mp.mpf(z[i])
            t2.append([float(mp.diff(lambda u: _sph_truth(kind, A, u), Bz, 2)),
                       float(mp.diff(lambda u, w: _sph_truth(kind, u, w), (A, Bz), (1, 1))),
                       float(mp.diff(lambda u: _sph_truth(kind, u, Bz), A, 2))])
        d[f"{name}_idx2"], d[f"{name}_truth2"] = idx, np.array(t2)
        d[f"{name}_ref"] = ref(name, 0, n, z)[0]
        d[f"{name}_ref_grad"] = np.stack(ref(name, 1, g, n, z), axis=1)
        sn = np.array([0.0, 1.0, 2.0, -0.5, 0.0, 1.0, 3.0, np.nan, 1.0])
        sz = np.array([0.0, 0.0, 1e-13, 0.0, -1e-13, -2.0, -2.0, 1.0, np.nan])
        d[f"{name}_special_n"], d[f"{name}_special_z"] = sn, sz
        d[f"{name}_special_ref"] = ref(name, 0, sn, sz)[0]
        d[f"{name}_special_ref_grad"] = np.stack(ref(name, 1, np.ones_like(sn), sn, sz), axis=1)
    np.savez_compressed(OUT / "spherical.npz", **d)


def _ibeta_truth(x, a, b):
    """I_x(a, b) and its first derivatives at 40 digits.  Where I > 1/2 the
    complement 1 - I_x(a, b) = I_(1-x)(b, a) is evaluated instead (its
    value and parameter derivatives keep their relative accuracy when they
    are tiny), and the a/b derivatives are its negatives."""
    X, A, B = mp.mpf(x), mp.mpf(a), mp.mpf(b)
    lo = mp.betainc(A, B, 0, X, regularized=True)
    comp = lo > 0.5
    if comp:
        f = lambda u, v: mp.betainc(v, u, 0, 1 - X, regularized=True)  # noqa: E731
        hi = f(A, B)
        val = 1 - hi
        da, db = -mp.diff(lambda u: f(u, B), A), -mp.diff(lambda v: f(A, v), B)
    else:
        f = lambda u, v: mp.betainc(u, v, 0, X, regularized=True)  # noqa: E731
        val = lo
        da, db = mp.diff(lambda u: f(u, B), A), mp.diff(lambda v: f(A, v), B)
    pdf = mp.exp((A - 1) * mp.log(X) + (B - 1) * mp.log1p(-X)) / mp.beta(A, B)
    return val, pdf, da, db, f, comp


def incomplete_beta():
    """incomplete_beta: seeded x in (0, 1), a and b log-uniform over
    [0.05, 300] (a block drawn near the swap line x = (a+1)/(a+b+2), a block
    with a or b near 1, a block of a, b in [300, 3000]); mpmath values (40
    digits) of I, ∂x, ∂a, ∂b and, on every tenth point, the six second
    derivatives; the reference's outputs; the reference's special points."""
    rng = np.random.default_rng(14)
    n = 600
    a = lu(rng, 0.05, 300.0, n)
    b = lu(rng, 0.05, 300.0, n)
    x = rng.uniform(0.0, 1.0, n)
    x[:100] = np.clip((a[:100] + 1) / (a[:100] + b[:100] + 2) * rng.uniform(0.9, 1.1, 100), 1e-6, 1 - 1e-6)
    a[100:130] = 1.0 + rng.uniform(-1e-3, 1e-3, 30)
    b[130:160] = 1.0 + rng.uniform(-1e-3, 1e-3, 30)
    a[160:200] = lu(rng, 300.0, 3000.0, 40)
    b[160:200] = lu(rng, 300.0, 3000.0, 40)
    x[160:200] = np.clip(a[160:200] / (a[160:200] + b[160:200]) + rng.normal(0, 0.02, 40), 1e-3, 1 - 1e-3)
    x[200:240] = lu(rng, 1e-8, 1e-2, 40)
    x[240:280] = 1 - lu(rng, 1e-8, 1e-2, 40)
    d = {"x": x, "a": a, "b": b, "g": rng.standard_normal(n)}
    cols = {k: [] for k in ("v", "dx", "da", "db")}
    idx2 = np.arange(0, n, 10)
    sec = {k: [] for k in ("hxx", "hxa", "hxb", "haa", "hab", "hbb")}
    for i in range(n):
        val, pdf, da, db, f, comp = _ibeta_truth(x[i], a[i], b[i])
        for k, v in zip(("v", "dx", "da", "db"), (val, pdf, da, db)):
            cols[k].append(float(v))
        if i in set(idx2.tolist()):
            X, A, B = mp.mpf(x[i]), mp.mpf(a[i]), mp.mpf(b[i])
            sgn = -1 if comp else 1
            sec["hxx"].append(float(pdf * ((A - 1) / X - (B - 1) / (1 - X))))
            sec["hxa"].append(float(pdf * (mp.log(X) - mp.digamma(A) + mp.digamma(A + B))))
            sec["hxb"].append(float(pdf * (mp.log1p(-X) - mp.digamma(B) + mp.digamma(A + B))))
            sec["haa"].append(float(sgn * mp.diff(lambda u, v: f(u, v), (A, B), (2, 0))))
            sec["hab"].append(float(sgn * mp.diff(lambda u, v: f(u, v), (A, B), (1, 1))))
            sec["hbb"].append(float(sgn * mp.diff(lambda u, v: f(u, v), (A, B), (0, 2))))
    for k, v in cols.items():
        d[f"truth_{k}"] = np.array(v)
    d["idx2"] = idx2
    for k, v in sec.items():
        d[f"truth_{k}"] = np.array(v)
    gg = rng.standard_normal((3, n))
    d["gg"] = gg
    d["ref"] = ref("incomplete_beta", 0, x, a, b)[0]
    d["ref_grad"] = np.stack(ref("incomplete_beta", 1, d["g"], x, a, b), axis=1)
    i2 = idx2
    d["ref_bb"] = np.stack(ref("incomplete_beta", 2, gg[0][i2], gg[1][i2], gg[2][i2], d["g"][i2], x[i2], a[i2], b[i2]), axis=1)
    sx = np.array([0.0, -0.5, 1.0, 1.5, 0.3, 0.3, 0.3, 0.3, 0.3, 0.4, 0.7, np.nan, 0.5, 0.5, 1e-300])
    sa = np.array([2.0, 2.0, 2.0, 2.0, 0.0, -1.0, 1.0, 1.0, 2.5, 2.5, 1.0, 2.0, np.nan, 3.0, 2.0])
    sb = np.array([3.0, 3.0, 3.0, 3.0, 2.0, 2.0, 1.0, 2.5, 1.0, 0.0, 3.0, 3.0, 2.0, np.nan, 3.0])
    d["special_x"], d["special_a"], d["special_b"] = sx, sa, sb
    d["special_ref"] = ref("incomplete_beta", 0, sx, sa, sb)[0]
    d["special_ref_grad"] = np.stack(ref("incomplete_beta", 1, np.ones_like(sx), sx, sa, sb), axis=1)
    np.savez_compressed(OUT / "incomplete_beta.npz", **d)


if __name__ == "__main__":
    which = sys.argv[1:] or ["gamma_family", "igamma", "elliptic", "bessel", "bessel01", "hyp2f1", "probability", "probability_density", "beta_family", "bessel_int", "spherical01", "spherical", "incomplete_beta"]
    for w in which:
        globals()[w]()
        print("wrote", w)
