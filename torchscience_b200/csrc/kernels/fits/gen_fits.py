"""Generates fits.cuh: polynomial fits used by the device evaluators.

Each fit is a Chebyshev interpolant of a smooth function on an interval,
computed with mpmath at 60 digits, converted to monomial coefficients in the
interval's scaled variable u in [-1, 1] and rounded to double.  The script
checks the double-precision Horner evaluation against mpmath on a dense grid
and prints the worst relative error of each fit.

    python torchscience_b200/csrc/kernels/fits/gen_fits.py

Fits:
  PSI_ROOT:  ψ(x) / (x - x0) on x in [1, 2] (x0 = positive root of ψ),
             u = 2x - 3.  ψ(x) = (x - x0) * P(u) has no cancellation near x0.
  LGAMMA1P:  lnΓ(1 + a) / a on a in [0, 1], u = 2a - 1 (value -γ at a = 0),
             so lnΓ(1 + a) keeps its absolute accuracy for small a without
             rounding 1 + a.
  TEMME_G1, TEMME_G2: the Γ combinations of Temme's series for Y_μ, K_μ
             (|μ| <= 1/2), u = 2μ:
               g1(μ) = (1/Γ(1-μ) - 1/Γ(1+μ)) / (2μ)   (limit -γ at μ = 0)
               g2(μ) = (1/Γ(1-μ) + 1/Γ(1+μ)) / 2
"""

from __future__ import annotations

from pathlib import Path

import mpmath as mp

mp.mp.dps = 60
OUT = Path(__file__).resolve().parent.parent / "fits.cuh"


def cheb_fit(f, n):
    """Chebyshev interpolation of f on [-1, 1] with n+1 nodes -> monomial coeffs in u."""
    nodes = [mp.cos(mp.pi * (k + mp.mpf(1) / 2) / (n + 1)) for k in range(n + 1)]
    vals = [f(u) for u in nodes]
    c = []
    for j in range(n + 1):
        s = mp.fsum(vals[k] * mp.cos(mp.pi * j * (k + mp.mpf(1) / 2) / (n + 1)) for k in range(n + 1))
        c.append(s * (1 if j == 0 else 2) / (n + 1))
    # Chebyshev -> monomial
    T = [[mp.mpf(1)], [mp.mpf(0), mp.mpf(1)]]
    for j in range(2, n + 1):
        t = [mp.mpf(0)] * (j + 1)
        for i, v in enumerate(T[j - 1]):
            t[i + 1] += 2 * v
        for i, v in enumerate(T[j - 2]):
            t[i] -= v
        T.append(t)
    mono = [mp.mpf(0)] * (n + 1)
    for j in range(n + 1):
        for i, v in enumerate(T[j]):
            mono[i] += c[j] * v
    return mono


def horner(coeffs, u):
    r = 0.0
    for c in reversed(coeffs):
        r = r * u + c
    return r


X0 = mp.findroot(mp.digamma, mp.mpf("1.4616321449683623"))


def psi_root_fn(u):
    x = mp.mpf(3) / 2 + u / 2
    if abs(x - X0) < mp.mpf("1e-40"):
        return mp.psi(1, X0)
    return mp.digamma(x) / (x - X0)


def lgamma1p_fn(u):
    a = (u + 1) / 2
    if a == 0:
        return -mp.euler
    return mp.loggamma(1 + a) / a


def temme_g1(u):
    mu = u / 2
    if abs(mu) < mp.mpf("1e-30"):
        return -mp.euler
    return (1 / mp.gamma(1 - mu) - 1 / mp.gamma(1 + mu)) / (2 * mu)


def temme_g2(u):
    mu = u / 2
    return (1 / mp.gamma(1 - mu) + 1 / mp.gamma(1 + mu)) / 2


def check(fn, coeffs, lo=-1.0, hi=1.0, n=4001):
    worst = 0.0
    for k in range(n):
        u = lo + (hi - lo) * k / (n - 1)
        want = fn(mp.mpf(u))
        got = horner([float(c) for c in coeffs], u)
        worst = max(worst, abs((got - want) / want))
    return float(worst)


def emit(name, coeffs, ctype):
    # Coefficients that vanish by symmetry come out ~1e-60; store them as 0.
    vals = ", ".join(repr(float(c) if abs(c) > 1e-40 else 0.0) + ("f" if ctype == "float" else "") for c in coeffs)
    return f"__device__ constexpr {ctype} {name}[{len(coeffs)}] = {{{vals}}};\n"


def main():
    x0_hi = float(X0)
    x0_lo = float(X0 - mp.mpf(x0_hi))
    import numpy as np

    x0f_hi = float(np.float32(x0_hi))
    x0f_lo = float(np.float32(float(X0 - mp.mpf(x0f_hi))))
    psi_d = cheb_fit(psi_root_fn, 26)
    psi_f = cheb_fit(psi_root_fn, 12)
    print("PSI_ROOT double worst rel err", check(psi_root_fn, psi_d))
    print("PSI_ROOT float  worst rel err", check(psi_root_fn, psi_f))
    g1_d, g2_d = cheb_fit(temme_g1, 22), cheb_fit(temme_g2, 22)
    g1_f, g2_f = cheb_fit(temme_g1, 10), cheb_fit(temme_g2, 10)
    print("TEMME_G1 double worst rel err", check(temme_g1, g1_d), "float", check(temme_g1, g1_f))
    print("TEMME_G2 double worst rel err", check(temme_g2, g2_d), "float", check(temme_g2, g2_f))
    lg1p_d = cheb_fit(lgamma1p_fn, 28)
    print("LGAMMA1P double worst rel err", check(lgamma1p_fn, lg1p_d, hi=0.99))
    text = (
        "// Generated by fits/gen_fits.py (mpmath Chebyshev interpolation); do not edit.\n"
        "#pragma once\n\nnamespace tsb {\nnamespace fits {\n\n"
        f"// Positive root of digamma, split hi + lo.\n"
        f"__device__ constexpr double PSI_X0_HI = {x0_hi!r};\n"
        f"__device__ constexpr double PSI_X0_LO = {x0_lo!r};\n"
        f"__device__ constexpr float PSI_X0_HI_F = {x0f_hi!r}f;\n"
        f"__device__ constexpr float PSI_X0_LO_F = {x0f_lo!r}f;\n"
        "// psi(x) / (x - x0) on [1, 2] as a polynomial in u = 2x - 3 (ascending powers).\n"
        + emit("PSI_ROOT_D", psi_d, "double")
        + emit("PSI_ROOT_F", psi_f, "float")
        + "// Temme's g1(μ) = (1/Γ(1-μ) - 1/Γ(1+μ))/(2μ), g2(μ) = (1/Γ(1-μ) + 1/Γ(1+μ))/2, |μ| <= 1/2, in u = 2μ.\n"
        + emit("TEMME_G1_D", g1_d, "double")
        + emit("TEMME_G2_D", g2_d, "double")
        + emit("TEMME_G1_F", g1_f, "float")
        + emit("TEMME_G2_F", g2_f, "float")
        + "// lnΓ(1 + a) / a on [0, 1] as a polynomial in u = 2a - 1.\n"
        + emit("LGAMMA1P_D", lg1p_d, "double")
        + "\n}  // namespace fits\n}  // namespace tsb\n"
    )
    OUT.write_text(text)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
