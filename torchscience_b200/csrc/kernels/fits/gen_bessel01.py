"""Generates bessel01_fits.cuh: J0 and J1 of real argument for the order-0/1 path.

    python torchscience_b200/csrc/kernels/fits/gen_bessel01.py

Two forms, both fitted with mpmath at 50 digits (Chebyshev interpolation,
converted to monomials in the interval's scaled variable u in [-1, 1]):

  Zero intervals, 0 <= x < X0 = 16.25π.  J0 interval i (1..16) covers
  [(i - 3/4)π, (i + 1/4)π) (interval 1 starts at 0) and holds the i-th zero
  z of J0; J1 interval i (0..16) covers [(i - 1/4)π, (i + 3/4)π) and holds
  the i-th zero of J1 (z = 0 for i = 0).  In each, J(x) = (x - z)·P(u): z is
  stored as a hi + lo pair, so x - z keeps its relative accuracy next to the
  zero and the value keeps full relative accuracy there.  The interval of x
  is floor(x/π + 3/4) (J0) or floor(x/π + 1/4) (J1); the fits cover each
  interval widened by 1/64 on both sides, so a rounded index is harmless.
  u = (x - c)·s is formed on the device from the stored doubles c and s, and
  the fit is made in exactly that variable.

  Modulus/phase form, x >= X0 (DLMF 10.17.3):
      J_n(x) = sqrt(2/(πx))·(P_n cos χ - Q_n sin χ),  χ = x - (2n + 1)π/4,
  with P_n and x·Q_n fitted as polynomials in 2t - 1, t = (X0/x)² on (0, 1].
  P_n, Q_n are computed from mpmath's J_n and Y_n, not from the divergent
  Hankel series.

The script checks every fit against mpmath on a dense grid in double
precision (Horner, as the device evaluates it) and prints the worst errors
(all below 5e-16 relative).
"""

from __future__ import annotations

from pathlib import Path

import mpmath as mp

mp.mp.dps = 50
OUT = Path(__file__).resolve().parent.parent / "bessel01_fits.cuh"

NI = 17  # intervals per function: J0 uses 1..16 (slot 0 is a copy of 1), J1 uses 0..16
X0 = 16.25 * float(mp.pi)  # rounded to double; every bound below uses this double
DEG_IV = 18
DEG_ASY = 7
WIDEN = 1.0 / 64


def cheb_mono(f, n):
    """Degree-n Chebyshev interpolant of f(u) on [-1, 1] as monomial coefficients in u."""
    nodes = [mp.cos(mp.pi * (k + mp.mpf(1) / 2) / (n + 1)) for k in range(n + 1)]
    vals = [f(u) for u in nodes]
    c = []
    for j in range(n + 1):
        s = mp.fsum(vals[k] * mp.cos(mp.pi * j * (k + mp.mpf(1) / 2) / (n + 1)) for k in range(n + 1))
        c.append(s * (1 if j == 0 else 2) / (n + 1))
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
    return [float(m) for m in mono]


def horner(cs, u):
    r = 0.0
    for c in reversed(cs):
        r = r * u + c
    return r


def interval(order, i):
    if order == 0:
        lo, hi = (0.0 if i == 1 else (i - 0.75) * float(mp.pi)), (i + 0.25) * float(mp.pi)
        z = mp.besseljzero(0, i)
    else:
        lo, hi = max(0.0, (i - 0.25) * float(mp.pi)), (i + 0.75) * float(mp.pi)
        z = mp.mpf(0) if i == 0 else mp.besseljzero(1, i)
    hi = min(hi, X0)
    assert lo < z < hi or (order == 1 and i == 0), (order, i, lo, z, hi)
    return lo - WIDEN, hi + WIDEN, z


def zero_fit(order, i):
    lo, hi, z = interval(order, i)

    def f(x):
        if abs(x - z) < mp.mpf("1e-30"):
            return mp.besselj(order, z, derivative=1)
        return mp.besselj(order, x) / (x - z)

    # The device forms u = (x - c)·s from the stored doubles c and s, so the
    # fit is made in exactly that variable (x = c + u/s in full precision).
    c, s = (lo + hi) / 2, 2 / (hi - lo)
    cs = cheb_mono(lambda u: f(mp.mpf(c) + u / mp.mpf(s)), DEG_IV)
    z_hi = float(z)
    z_lo = float(z - mp.mpf(z_hi))
    # check: relative error of (x - z)·P(u) in double against mpmath
    worst = 0.0
    for k in range(1201):
        x = lo + (hi - lo) * k / 1200
        if x < 0:
            continue
        want = mp.besselj(order, x)
        got = ((x - z_hi) - z_lo) * horner(cs, (x - c) * s)
        if want != 0:
            worst = max(worst, float(abs((got - want) / want)))
    return cs, c, s, z_hi, z_lo, worst


def pq(order, x):
    x = mp.mpf(x)
    chi = x - (2 * order + 1) * mp.pi / 4
    j, y = mp.besselj(order, x), mp.bessely(order, x)
    k = mp.sqrt(mp.pi * x / 2)
    return k * (j * mp.cos(chi) + y * mp.sin(chi)), k * (y * mp.cos(chi) - j * mp.sin(chi))


def asy_fits(order):
    def p(tu):  # tu in [-1, 1] -> t in [0, 1]
        t = (tu + 1) / 2
        if t == 0:
            return mp.mpf(1)
        return pq(order, X0 / mp.sqrt(t))[0]

    def xq(tu):
        t = (tu + 1) / 2
        if t == 0:
            return mp.mpf(4 * order * order - 1) / 8
        x = X0 / mp.sqrt(t)
        return x * pq(order, x)[1]

    cp = cheb_mono(p, DEG_ASY)
    cq = cheb_mono(xq, DEG_ASY)
    wp = wq = 0.0
    for k in range(1, 801):
        t = k / 800
        x = X0 / mp.sqrt(t)
        P, Q = pq(order, x)
        wp = max(wp, float(abs(horner(cp, 2 * t - 1) - P) / abs(P)))
        wq = max(wq, float(abs(horner(cq, 2 * t - 1) / x - Q) / abs(Q)))
    return cp, cq, wp, wq


def fmt(v):
    return repr(float(v))


def main():
    tabs = {}
    for order in (0, 1):
        rows = []
        for i in range(NI):
            if order == 0 and i == 0:
                rows.append(None)
                continue
            cs, c, s, zh, zl, w = zero_fit(order, i)
            print(f"J{order} interval {i:2d}: worst rel err {w:.2e}")
            rows.append((cs, c, s, zh, zl))
        rows[0] = rows[0] or rows[1]  # J0 slot 0 is never indexed; keep it a valid copy
        tabs[order] = rows
    asy = {}
    for order in (0, 1):
        cp, cq, wp, wq = asy_fits(order)
        print(f"J{order} asymptotic: P worst rel {wp:.2e}, Q worst rel {wq:.2e}")
        asy[order] = (cp, cq)

    out = [
        "// Generated by fits/gen_bessel01.py (mpmath Chebyshev interpolation); do not edit.\n",
        "#pragma once\n\nnamespace tsb {\nnamespace fits {\n\n",
        f"constexpr int B01_NI = {NI};\n",
        f"constexpr int B01_DEG = {DEG_IV};\n",
        f"constexpr double B01_X0 = {fmt(X0)};  // 16.25π rounded to double\n",
        f"constexpr double B01_X0_SQ = {fmt(X0 * X0)};\n\n",
    ]
    for order in (0, 1):
        rows = tabs[order]
        out.append(f"// J{order}: per interval {{center, 1/half-width, zero hi, zero lo}}.\n")
        out.append(f"__device__ const double B01_J{order}_IV[{NI}][4] = {{\n")
        for r in rows:
            out.append(f"    {{{fmt(r[1])}, {fmt(r[2])}, {fmt(r[3])}, {fmt(r[4])}}},\n")
        out.append("};\n")
        out.append(f"// J{order}(x)/(x - z) as a polynomial in u: coefficient k of interval i at [k][i].\n")
        out.append(f"__device__ const double B01_J{order}_C[{DEG_IV + 1}][{NI}] = {{\n")
        for k in range(DEG_IV + 1):
            out.append("    {" + ", ".join(fmt(r[0][k]) for r in rows) + "},\n")
        out.append("};\n\n")
    for order in (0, 1):
        cp, cq = asy[order]
        out.append(f"// P{order}(t) and x·Q{order}(t), t = (X0/x)², ascending powers of 2t - 1.\n")
        out.append(f"__device__ constexpr double B01_P{order}[{DEG_ASY + 1}] = {{" + ", ".join(fmt(c) for c in cp) + "};\n")
        out.append(f"__device__ constexpr double B01_Q{order}[{DEG_ASY + 1}] = {{" + ", ".join(fmt(c) for c in cq) + "};\n")
    out.append("\n}  // namespace fits\n}  // namespace tsb\n")
    OUT.write_text("".join(out))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
