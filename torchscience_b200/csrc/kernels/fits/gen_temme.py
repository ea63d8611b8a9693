"""Generates temme_fits.cuh: the coefficients of Temme's uniform asymptotic
expansion of the regularized incomplete gamma functions (DLMF 8.12.3-8.12.4,
8.12.10), for the transition x ~ a at large a.

    python torchscience_b200/csrc/kernels/fits/gen_temme.py

With λ = x/a and η = sign(λ-1)·sqrt(2(λ - 1 - ln λ)),
    Q(a, x) = ½ erfc(η sqrt(a/2)) + R_a(η),   P = 1 - Q,
    R_a(η) ~ exp(-aη²/2) / sqrt(2πa) · Σ_k c_k(η) a^-k,
    c_0(η) = 1/(λ-1) - 1/η,
    c_k(η) = (1/η) c'_{k-1}(η) + (-1)^k g_k / (λ-1),
where g_k are the coefficients of Γ*(a) = Γ(a)/(sqrt(2π) e^-a a^(a-½))
~ Σ g_k a^-k (DLMF 5.11.3; here from its logarithm, Σ B_2m / (2m(2m-1) a^(2m-1))).
Each c_k is analytic at η = 0 (the 1/η terms cancel); this script works with
their Taylor series, in mpmath at 80 digits:
  1. λ - 1 = u(η) by reversing η(u) = u sqrt(2(u - ln(1+u))/u²);
  2. 1/(λ-1) = (1/η)·1/(u/η), so c_0 and every c_k are series in η;
  3. each c_k is truncated where its terms fall below 1e-20 of the sum's scale
     on the range the kernels use it (a >= TEMME_A_MIN, |η| <= TEMME_ETA_MAX).
The script checks the truncated expansion, evaluated in double precision by
Horner as the device does, against mpmath's incomplete gamma on a grid of
(a, λ) in that range, and prints the worst relative errors of Q (or P) and of
∂P/∂a.
"""

from __future__ import annotations

import os

import mpmath as mp
import numpy as np

mp.mp.dps = 80
N = 48          # Taylor terms carried during generation
K = 9           # terms in 1/a: c_0 .. c_{K-1}
A_MIN = 100.0
ETA_MAX = 0.52  # |η| at λ = 0.6 and λ = 1.6
LAM_LO, LAM_HI = 0.6, 1.6
TOL = 1e-20


def mul(a, b):
    c = [mp.mpf(0)] * N
    for i, ai in enumerate(a):
        if ai == 0:
            continue
        for j in range(N - i):
            c[i + j] += ai * b[j]
    return c


def inv(a):
    b = [mp.mpf(0)] * N
    b[0] = 1 / a[0]
    for n in range(1, N):
        b[n] = -sum(a[k] * b[n - k] for k in range(1, n + 1)) / a[0]
    return b


def sqrt1(a):  # sqrt of a series with a[0] = 1
    b = [mp.mpf(0)] * N
    b[0] = mp.mpf(1)
    for n in range(1, N):
        b[n] = (a[n] - sum(b[k] * b[n - k] for k in range(1, n))) / 2
    return b


def compose(f, g):  # f(g(t)) with g[0] = 0
    res = [mp.mpf(0)] * N
    p = [mp.mpf(0)] * N
    p[0] = mp.mpf(1)
    for k in range(N):
        if k > 0:
            p = mul(p, g)
        if f[k] != 0:
            for i in range(N):
                res[i] += f[k] * p[i]
    return res


def coefficients():
    t = [mp.mpf(2) * (-1) ** n / n for n in range(2, N + 2)]   # 2(u - ln(1+u))/u², n - 2 = power
    eta_u = [mp.mpf(0)] + sqrt1(t)[: N - 1]                     # η as a series in u
    u = [mp.mpf(0)] * N
    u[1] = mp.mpf(1)
    for _ in range(N):                                           # u(η) by fixed-point reversion
        e = compose(eta_u, u)
        u = [u[i] - (e[i] - (1 if i == 1 else 0)) for i in range(N)]
    ue = u[1:] + [mp.mpf(0)]                                     # u/η
    inv_ue = inv(ue)                                             # η/u;  1/u = inv_ue / η
    L = [mp.mpf(0)] * N                                          # ln Γ*(a) in powers of 1/a
    for m in range(1, N // 2):
        L[2 * m - 1] = mp.bernoulli(2 * m) / (2 * m * (2 * m - 1))
    g = [mp.mpf(0)] * N                                          # Γ*(a) = exp(L)
    g[0] = mp.mpf(1)
    for n in range(1, N):
        g[n] = sum(k * L[k] * g[n - k] for k in range(1, n + 1)) / n
    C = [inv_ue[1:] + [mp.mpf(0)]]                               # c_0 = (η/u - 1)/η
    for k in range(1, K):
        d = [(i + 1) * C[-1][i + 1] for i in range(N - 1)] + [mp.mpf(0)]
        num = [d[i] + (-1) ** k * g[k] * inv_ue[i] for i in range(N)]
        assert abs(num[0]) < mp.mpf(10) ** -60, (k, num[0])     # the 1/η terms cancel
        C.append(num[1:] + [mp.mpf(0)])
    return C, ue


def truncate(C, ue):
    out = []
    for k, c in enumerate(C):
        scale = mp.mpf(A_MIN) ** -k
        n = N
        while n > 1 and all(abs(c[j]) * mp.mpf(ETA_MAX) ** j * scale < TOL for j in range(n - 1, N)):
            n -= 1
        out.append([float(v) for v in c[:n]])
    nue = N
    while nue > 1 and all(abs(ue[j]) * mp.mpf(ETA_MAX) ** j < 1e-20 for j in range(nue - 1, N)):
        nue -= 1
    return out, [float(v) for v in ue[:nue]]  # u/η as a series: the check's dη/da


def horner(c, x):
    s = 0.0
    for v in reversed(c):
        s = s * x + v
    return s


def dhorner(c, x):  # derivative of the series
    s = 0.0
    for j in range(len(c) - 1, 0, -1):
        s = s * x + j * c[j]
    return s


def evaluate(a, x, Ck, UE):
    """Q and dP/da in double precision, as the device evaluates them."""
    import math

    u = (x - a) / a
    lm = math.log1p(u) - u
    eta = math.copysign(math.sqrt(-2.0 * lm), u) if u != 0 else 0.0
    S = Sa = Se = 0.0
    ra = 1.0 / a
    for k in range(len(Ck) - 1, -1, -1):
        S = S * ra + horner(Ck[k], eta)
        Se = Se * ra + dhorner(Ck[k], eta)
        Sa = Sa * ra + k * horner(Ck[k], eta)
    Sa = -Sa * ra
    pref = math.exp(a * lm) / math.sqrt(2.0 * math.pi * a)
    s = eta * math.sqrt(0.5 * a)
    R = pref * S
    # the smaller of P and Q directly, the other as 1 minus it
    small = 0.5 * math.erfc(s) + R if eta >= 0.0 else 0.5 * math.erfc(-s) - R
    rue = horner(UE, eta)
    dpda = pref * (0.5 * eta - rue - S * (math.log1p(u) - 0.5 * ra) - Sa + Se * rue * ra)
    return small, dpda


def check(Ck, UE):
    worst_v = worst_d = 0.0
    at_v = at_d = None
    for a in (100.0, 131.7, 200.0, 511.0, 1000.0, 4096.0, 1e5):
        for lam in np.linspace(LAM_LO, LAM_HI, 41):
            x = a * lam
            got_small, dpda = evaluate(a, x, Ck, UE)
            am, xm = mp.mpf(a), mp.mpf(x)
            Q = mp.gammainc(am, xm, mp.inf, regularized=True)
            P = 1 - Q
            small = min(P, Q)
            if small < mp.mpf("1e-300"):  # below the double range: the kernels saturate there
                continue
            ev = float(abs(got_small - small) / small)
            if ev > worst_v:
                worst_v, at_v = ev, (a, lam)
            worst_v = max(worst_v, ev)
            # differentiate the smaller of P and Q (the other is 1 minus it, beyond 80 digits' reach)
            if Q <= P:
                dP = -mp.diff(lambda s: mp.gammainc(s, xm, mp.inf, regularized=True), am)
            else:
                dP = mp.diff(lambda s: mp.gammainc(s, 0, xm, regularized=True), am)
            if abs(dP) > mp.mpf("1e-300"):
                ed = float(abs(dpda - dP) / abs(dP))
                if ed > worst_d:
                    worst_d, at_d = ed, (a, lam)
    print("worst at", at_v, at_d)
    return worst_v, worst_d


def main():
    C, ue = coefficients()
    Ck, UE = truncate(C, ue)
    wv, wd = check(Ck, UE)
    print(f"terms per c_k: {[len(c) for c in Ck]}, u/eta terms: {len(UE)}")
    print(f"worst relative error of min(P, Q): {wv:.3e}; of dP/da: {wd:.3e}")
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "temme_fits.cuh")
    lines = ["// Generated by fits/gen_temme.py (mpmath, 80 digits); do not edit.", "#pragma once", "",
             "namespace tsb {", "namespace fits {", "",
             f"constexpr double TEMME_A_MIN = {A_MIN!r};", f"constexpr double TEMME_LAM_LO = {LAM_LO!r};",
             f"constexpr double TEMME_LAM_HI = {LAM_HI!r};", f"constexpr int TEMME_K = {len(Ck)};", ""]
    lines += ["// S = Σ_k c_k(η) r^k with r = 1/a; when DERIV also Se = Σ_k c_k'(η) r^k and",
              "// Sk = Σ_k k c_k(η) r^k (so that ∂S/∂a = -r Sk).  Horner in η for each c_k (and its",
              "// derivative), then in r, written out with the coefficients as constants: the",
              "// evaluation is its FMAs alone, about two per coefficient.",
              "template <bool DERIV>",
              "__device__ __forceinline__ void temme_sums(double eta, double r, double& S, double& Se, double& Sk) {",
              "  double c, d;",
              "  S = Se = Sk = 0.0;"]
    for k in range(len(Ck) - 1, -1, -1):
        c = Ck[k]
        lines.append(f"  // c_{k}: {len(c)} terms")
        lines.append(f"  c = {c[-1]!r};")
        lines.append("  d = 0.0;")
        for j in range(len(c) - 2, -1, -1):
            lines.append(f"  if (DERIV) d = fma(d, eta, c);")
            lines.append(f"  c = fma(c, eta, {c[j]!r});")
        lines.append("  S = fma(S, r, c);")
        lines.append("  if (DERIV) {")
        lines.append("    Se = fma(Se, r, d);")
        if k:
            lines.append(f"    Sk = fma(Sk, r, {float(k)!r} * c);")
        else:
            lines.append("    Sk = Sk * r;")
        lines.append("  }")
    lines.append("}")

    lines += ["", "}  // namespace fits", "}  // namespace tsb", ""]
    open(path, "w").write("\n".join(lines))
    print("wrote", path)


if __name__ == "__main__":
    main()
