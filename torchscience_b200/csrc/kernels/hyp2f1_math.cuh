// Gauss hypergeometric function 2F1(a, b; c; z) for real arguments, z < 1,
// with its first and second derivatives.
//
// Special cases follow the reference in its order (hypergeometric_2_f_1.h:203-295):
// z ~ 0 or a ~ 0 or b ~ 0 -> 1; c a non-positive integer -> +inf unless a or
// b terminates the series first; |z| = 1 (z != 1) with c - a - b <= -1 ->
// NaN; c ~ b -> (1-z)^-a; c ~ a -> (1-z)^-b; a or b a non-positive integer
// -> the terminating polynomial; z ~ 1 -> Gauss's sum Γ(c)Γ(c-a-b) /
// (Γ(c-a)Γ(c-b)) (NaN if c - a - b <= 0); z > 1 -> NaN.
//
// Elsewhere the reference sums the series (hypergeometric_2_f_1.h:75-94)
// directly for 0 <= z < 1/2, Pfaff-transformed for z < 0 (:151-163), and
// with 2000 terms of the direct series for 1/2 <= z < 1 (:96-116), which
// has not converged near z = 1.  Here every evaluation is of
// G(p, q; c; x) for 0 <= x < 1, after the Pfaff transformation for z < 0:
//   F(a, b; c; z) = (1-z)^-a G(a, c-b; c; z/(z-1))   (or a <-> b);
// G is the direct series for x <= 1/2.  For x > 1/2 it is the 1 - x
// connection formula (DLMF 15.8.4), whose series run at 1 - x < 1/2, unless
// that formula's error estimate (ε Σ|terms|, its two terms cancel when
// c - p - q is near an integer) is larger than that of the direct series
// at x, in which case the direct series is used; when both are poor and
// c - p - q is within 1e-5 of an integer, the connection formula is
// evaluated at shifted c and extrapolated back.
// Derivatives in a, b, c are analytic in all cases: term-wise series
// derivatives (harmonic sums Σ 1/(p + k)) and, in the connection formula,
// derivatives of its Γ-ratios through ψ.  ∂/∂z comes from the same pass
// (d t_k/dx = k t_k/x, and the chain rule through the transformations); at
// the special points and for grad_z alone it is (ab/c) 2F1(a+1, b+1; c+1; z).
// Second derivatives in a, b, c are Richardson-extrapolated central
// differences of the analytic gradient (evaluator held fixed); those in z come
// from the gradient of 2F1(a+1, b+1; c+1; z).  At the special points the
// parameter derivatives are differences of the value, as in the reference
// (hypergeometric_2_f_1_backward.h:87-104): steps ε^(1/3) for the gradient
// and ε^(1/4) for the Hessian, scaled by max(1, |p|).
#pragma once

#include <math_constants.h>

#include "gamma_math.cuh"

namespace tsb {

// The large evaluators below are kept out of line (__noinline__): every
// kernel of a translation unit then shares one copy, which bounds code size,
// compile time and register pressure of the backward kernels.

constexpr double kH2f1Eps = 1e-15;  // the reference's parameter tolerance (hyp2f1_epsilon<double>)
constexpr double kH2Ulp = 1.1102230246251565e-16;
constexpr int kH2ConnTerms = 600;     // series at 1 - x <= 1/2
constexpr int kH2DirectTerms = 3000;  // direct series at x in (1/2, 1)

__device__ __forceinline__ bool h2f1_nonpos_int(double v, double eps = kH2f1Eps) {
  return v <= 0.0 && fabs(v - rint(v)) < eps;
}

// 1/Γ(x) and its derivative -ψ(x)/Γ(x), both finite at the poles of Γ:
// at x = -n, 1/Γ = 0 and d(1/Γ)/dx = (-1)^n n!.
__device__ inline double rgamma_d(double x) {
  if (x <= 0.0 && x == floor(x)) return 0.0;
  return 1.0 / tgamma(x);
}
__device__ inline void rgamma_dd(double x, double& r, double& dr) {
  if (x <= 0.0 && x == floor(x)) {
    r = 0.0;
    const double n = -x;
    dr = (fmod(n, 2.0) == 0.0 ? 1.0 : -1.0) * tgamma(n + 1.0);
    return;
  }
  r = 1.0 / tgamma(x);
  dr = -digamma_d(x) * r;
}

// Σ_k (p)_k (q)_k / ((c)_k k!) x^k with Σ|terms| and, if DERIVS, the
// derivatives in p, q, c and x (d t_k / dx = k t_k / x).  Convergence is
// tested only once k is past max(|p|, |q|), against the absolute sums (the
// attainable accuracy).
struct H2Sum {
  double s, abs, last;
  double dp, dq, dc, dx;
  bool conv;
};
template <bool DERIVS>
__device__ __noinline__ H2Sum h2f1_sum(double p, double q, double c, double x, int max_terms) {
  H2Sum r;
  double t = 1.0, s = 1.0, A = 1.0, hp = 0.0, hq = 0.0, hc = 0.0;
  double dp = 0.0, dq = 0.0, dc = 0.0, Ap = 0.0, Aq = 0.0, Ac = 0.0, kt = 0.0;
  const double kmin = fmax(fabs(p), fabs(q)) + 2.0;
  r.conv = false;
  for (int k = 0; k < max_terms; ++k) {
    const double fk = (double)k;
    const double pk = p + fk, qk = q + fk, ck = c + fk;
    if (DERIVS) {
      // one reciprocal per term: r = 1/(pk qk ck (k+1)) gives 1/pk, 1/qk, 1/ck
      // and the term ratio pk qk/(ck (k+1)) = (pk qk)^2 r
      const double pq = pk * qk, ck1 = ck * (fk + 1.0);
      const double r = 1.0 / (pq * ck1);
      hp = fma(qk * ck1, r, hp);
      hq = fma(pk * ck1, r, hq);
      hc = fma(pq * (fk + 1.0), r, hc);
      t *= pq * pq * r * x;
    } else {
      t *= pk * qk / (ck * (fk + 1.0)) * x;
    }
    s += t;
    A += fabs(t);
    if (DERIVS) {
      const double tp = t * hp, tq = t * hq, tc = t * hc;
      dp += tp;
      dq += tq;
      dc -= tc;
      kt = fma(fk + 1.0, t, kt);
      Ap += fabs(tp);
      Aq += fabs(tq);
      Ac += fabs(tc);
    }
    if (t == 0.0 || (fk > kmin && fabs(t) <= 0.25 * kH2Ulp * A)) {
      if (!DERIVS || t == 0.0 ||
          (fabs(t * hp) <= 0.25 * kH2Ulp * Ap && fabs(t * hq) <= 0.25 * kH2Ulp * Aq &&
           fabs(t * hc) <= 0.25 * kH2Ulp * Ac)) {
        r.conv = true;
        break;
      }
    }
  }
  r.s = s;
  r.abs = A;
  r.last = fabs(t);
  r.dp = dp;
  r.dq = dq;
  r.dc = dc;
  r.dx = DERIVS ? (x != 0.0 ? kt / x : p * q / c) : 0.0;
  return r;
}

// G(p, q; c; x) with an error estimate and, if DERIVS, its p-, q-, c- and
// x-derivatives.
struct H2Val {
  double v, err, dp, dq, dc, dx;
};

// Direct series; the estimate adds the truncated tail when not converged.
template <bool DERIVS>
__device__ inline H2Val h2f1_direct(double p, double q, double c, double x, int max_terms) {
  const H2Sum S = h2f1_sum<DERIVS>(p, q, c, x, max_terms);
  H2Val r;
  r.v = S.s;
  r.err = 4.0 * kH2Ulp * S.abs + (S.conv ? 0.0 : S.last * x / (1.0 - x));
  r.dp = S.dp;
  r.dq = S.dq;
  r.dc = S.dc;
  r.dx = S.dx;
  return r;
}

// The 1 - x connection formula, y = 1 - x in (0, 1/2]:
//   G = Γ(c)Γ(s)/(Γ(c-p)Γ(c-q)) F(p, q; 1-s; y)
//     + Γ(c)Γ(-s)/(Γ(p)Γ(q)) y^s F(c-p, c-q; 1+s; y),   s = c - p - q.
template <bool DERIVS>
__device__ __noinline__ H2Val h2f1_connect(double p, double q, double c, double y) {
  const double s = c - p - q, u = c - p, v = c - q;
  const double gc = tgamma(c), gs = tgamma(s), gms = tgamma(-s);
  double Pu, Du, Pv, Dv, Pp, Dp, Pq, Dq;
  if (DERIVS) {
    rgamma_dd(u, Pu, Du);
    rgamma_dd(v, Pv, Dv);
    rgamma_dd(p, Pp, Dp);
    rgamma_dd(q, Pq, Dq);
  } else {
    Pu = rgamma_d(u);
    Pv = rgamma_d(v);
    Pp = rgamma_d(p);
    Pq = rgamma_d(q);
    Du = Dv = Dp = Dq = 0.0;
  }
  const double ly = log(y), Y = exp(s * ly);
  const double G1 = gc * gs * Pu * Pv, G2 = gc * gms * Pp * Pq;
  H2Sum S1, S2;
  S1.s = S2.s = 1.0;
  S1.abs = S2.abs = 1.0;
  S1.dp = S1.dq = S1.dc = S1.dx = S2.dp = S2.dq = S2.dc = S2.dx = 0.0;
  S1.conv = S2.conv = true;
  if (G1 != 0.0 || DERIVS) S1 = h2f1_sum<DERIVS>(p, q, 1.0 - s, y, kH2ConnTerms);
  if (G2 != 0.0 || DERIVS) S2 = h2f1_sum<DERIVS>(u, v, 1.0 + s, y, kH2ConnTerms);
  H2Val r;
  const double T1 = G1 * S1.s, T2 = G2 * Y * S2.s;
  r.v = T1 + T2;
  // tgamma and the prefactor products add a few ulp to each term
  r.err = 8.0 * kH2Ulp * (fabs(G1) * S1.abs + fabs(G2 * Y) * S2.abs);
  if (!isfinite(r.v) || !(S1.conv || G1 == 0.0) || !(S2.conv || G2 == 0.0)) r.err = CUDART_INF;
  r.dp = r.dq = r.dc = r.dx = 0.0;
  if (DERIVS) {
    // d/dx = -d/dy: G1 S1'(y) + G2 y^s (s/y S2 + S2'(y))
    r.dx = -(G1 * S1.dx + G2 * Y * (s / y * S2.s + S2.dx));
    // s_p = s_q = -1, s_c = 1; u_p = -1, u_c = 1; v_q = -1, v_c = 1.
    const double psc = digamma_d(c), pss = digamma_d(s), psms = digamma_d(-s);
    const double gg1 = gc * gs, gg2 = gc * gms;
    const double G1p = gg1 * (-pss * Pu * Pv - Du * Pv);
    const double G1q = gg1 * (-pss * Pu * Pv - Pu * Dv);
    const double G1c = gg1 * ((psc + pss) * Pu * Pv + Du * Pv + Pu * Dv);
    const double G2p = gg2 * (psms * Pp * Pq + Dp * Pq);
    const double G2q = gg2 * (psms * Pp * Pq + Pp * Dq);
    const double G2c = gg2 * ((psc - psms) * Pp * Pq);
    // S1 = F(p, q; 1 - s; y): ∂(1 - s)/∂(p, q, c) = (1, 1, -1)
    const double S1p = S1.dp + S1.dc, S1q = S1.dq + S1.dc, S1c = -S1.dc;
    // S2 = F(u, v; 1 + s; y)
    const double S2p = -S2.dp - S2.dc, S2q = -S2.dq - S2.dc, S2c = S2.dp + S2.dq + S2.dc;
    r.dp = G1p * S1.s + G1 * S1p + Y * (G2p * S2.s - ly * G2 * S2.s + G2 * S2p);
    r.dq = G1q * S1.s + G1 * S1q + Y * (G2q * S2.s - ly * G2 * S2.s + G2 * S2q);
    r.dc = G1c * S1.s + G1 * S1c + Y * (G2c * S2.s + ly * G2 * S2.s + G2 * S2c);
  }
  return r;
}

// The connection formula with c shifted: when s = c - p - q is within about
// 1e-5 of an integer its two terms grow like 1/dist(s, Z) and cancel (and at
// an integer each is infinite).  G is analytic in c, so it is evaluated at
// c ± h and c ± 2h, where the formula is well conditioned, and the symmetric
// means m(h) are Richardson-extrapolated: G ≈ (4 m(h) - m(2h)) / 3, error
// O(h^4).  h = 1e-4, kept below 1/8 of the distance to a pole of Γ(c).
template <bool DERIVS>
__device__ inline H2Val h2f1_connect_shifted(double p, double q, double c, double y) {
  double h = 1e-4;
  if (c < 0.5) h = fmin(h, fabs(c - rint(c)) * 0.125);
  const H2Val r1 = h2f1_connect<DERIVS>(p, q, c + h, y), r2 = h2f1_connect<DERIVS>(p, q, c - h, y);
  const H2Val r3 = h2f1_connect<DERIVS>(p, q, c + 2.0 * h, y), r4 = h2f1_connect<DERIVS>(p, q, c - 2.0 * h, y);
  H2Val r;
  r.v = (2.0 * (r1.v + r2.v) - 0.5 * (r3.v + r4.v)) / 3.0;
  r.dp = (2.0 * (r1.dp + r2.dp) - 0.5 * (r3.dp + r4.dp)) / 3.0;
  r.dq = (2.0 * (r1.dq + r2.dq) - 0.5 * (r3.dq + r4.dq)) / 3.0;
  r.dc = (2.0 * (r1.dc + r2.dc) - 0.5 * (r3.dc + r4.dc)) / 3.0;
  r.dx = (2.0 * (r1.dx + r2.dx) - 0.5 * (r3.dx + r4.dx)) / 3.0;
  r.err = 2.0 * (r1.err + r2.err + r3.err + r4.err);
  return r;
}

// Evaluator for G at x in [0, 1): 0 direct series (x <= 1/2), 1 connection
// formula, 2 direct series at x > 1/2, 3 connection formula with c shifted.
enum H2Method : int { kH2mSeries = 0, kH2mConnect = 1, kH2mDirect = 2, kH2mShifted = 3 };

template <bool DERIVS>
__device__ inline H2Val h2f1_core(int method, double p, double q, double c, double x) {
  if (method == kH2mSeries) return h2f1_direct<DERIVS>(p, q, c, x, kH2ConnTerms);
  if (method == kH2mConnect) return h2f1_connect<DERIVS>(p, q, c, 1.0 - x);
  if (method == kH2mShifted) return h2f1_connect_shifted<DERIVS>(p, q, c, 1.0 - x);
  return h2f1_direct<DERIVS>(p, q, c, x, kH2DirectTerms);
}

enum H2f1Region : int {
  kH2Special = 0,
  kH2Series = 1,        // 0 <= z <= 1/2
  kH2Pfaff = 2,         // -1 <= z < 0
  kH2Connect = 3,       // 1/2 < z < 1
  kH2PfaffConnect = 4,  // z < -1
  kH2Regions = 5
};

// Terminating series (n terms after the first).
__device__ inline double h2f1_poly(double a, double b, double c, double z, int n) {
  double t = 1.0, s = 1.0;
  for (int k = 0; k < n; ++k) {
    const double fk = (double)k;
    t *= (a + fk) * (b + fk) / ((c + fk) * (fk + 1.0)) * z;
    s += t;
  }
  return s;
}

// The reference's early returns; true (with the value in v when VALUE) if
// (a, b, c, z) is one of them.  eps is the reference's parameter tolerance
// for the data type (hyp2f1_epsilon: 1e-15 for double, 1e-7 otherwise).
template <bool VALUE>
__device__ inline bool h2f1_special_t(double a, double b, double c, double z, double& v, double eps = kH2f1Eps) {
  if (isnan(a) || isnan(b) || isnan(c) || isnan(z)) {
    if (VALUE) v = CUDART_NAN;
    return true;
  }
  if (fabs(z) < eps || fabs(a) < eps || fabs(b) < eps) {
    if (VALUE) v = 1.0;
    return true;
  }
  if (h2f1_nonpos_int(c, eps)) {
    const double ci = rint(c);
    const bool a_cancels = h2f1_nonpos_int(a, eps) && rint(a) > ci;
    const bool b_cancels = h2f1_nonpos_int(b, eps) && rint(b) > ci;
    if (!a_cancels && !b_cancels) {
      if (VALUE) v = CUDART_INF;
      return true;
    }
  }
  if (fabs(fabs(z) - 1.0) < 1e-10 && !(fabs(z - 1.0) < 1e-10) && c - a - b <= -1.0) {
    if (VALUE) v = CUDART_NAN;
    return true;
  }
  if (fabs(c - b) < eps) {
    if (VALUE) v = pow(1.0 - z, -a);
    return true;
  }
  if (fabs(c - a) < eps) {
    if (VALUE) v = pow(1.0 - z, -b);
    return true;
  }
  if (h2f1_nonpos_int(a, eps)) {
    if (VALUE) v = h2f1_poly(a, b, c, z, -(int)rint(a));
    return true;
  }
  if (h2f1_nonpos_int(b, eps)) {
    if (VALUE) v = h2f1_poly(a, b, c, z, -(int)rint(b));
    return true;
  }
  if (fabs(z - 1.0) < 1e-10) {
    if (VALUE) {
      const double s = c - a - b;
      v = s <= 0.0 ? CUDART_NAN : tgamma(c) * tgamma(s) * rgamma_d(c - a) * rgamma_d(c - b);
    }
    return true;
  }
  if (z >= 1.0 || isinf(z) || isinf(a) || isinf(b) || isinf(c)) {
    if (VALUE) v = CUDART_NAN;
    return true;
  }
  return false;
}
__device__ inline bool h2f1_special(double a, double b, double c, double z, double& v, double eps = kH2f1Eps) {
  return h2f1_special_t<true>(a, b, c, z, v, eps);
}

__device__ __forceinline__ int h2f1_region_of(double z) {
  if (z >= 0.0) return z <= 0.5 ? kH2Series : kH2Connect;
  return z >= -1.0 ? kH2Pfaff : kH2PfaffConnect;
}

__device__ __forceinline__ int h2f1_classify(double a, double b, double c, double z, double eps = kH2f1Eps) {
  double v;
  if (h2f1_special_t<false>(a, b, c, z, v, eps)) return kH2Special;
  return h2f1_region_of(z);
}

// The Pfaff variant for z < 0: F = (1-z)^-p G(p, q; c; z/(z-1)) with
// (p, q) = (a, c - b), or (b, c - a) when swapped.
struct H2Plan {
  double p, q, x, lz;
  bool pfaff, swap;
  int method;
};
__device__ inline void h2f1_set_swap(H2Plan& P, double a, double b, double c, bool swap) {
  P.swap = swap;
  P.p = swap ? b : a;
  P.q = swap ? c - a : c - b;
}
__device__ inline H2Plan h2f1_plan(int region, double a, double b, double c, double z) {
  H2Plan P;
  P.pfaff = region == kH2Pfaff || region == kH2PfaffConnect;
  P.lz = 0.0;
  if (P.pfaff) {
    h2f1_set_swap(P, a, b, c, fabs(b * (c - a)) < fabs(a * (c - b)));
    P.x = z / (z - 1.0);
    P.lz = log1p(-z);
  } else {
    P.swap = false;
    P.p = a;
    P.q = b;
    P.x = z;
  }
  P.method = P.x <= 0.5 ? kH2mSeries : kH2mConnect;
  return P;
}

// Value at a non-special point.  The evaluator for x > 1/2 and, after the
// Pfaff transformation, the variant of the direct series are chosen here by
// the smallest relative error estimate; a first choice whose estimate is
// within 64 ulp is kept without trying the others.  The connection formula
// has the same relative error for both Pfaff variants.
static __device__ __noinline__ double h2f1_eval(int region, double a, double b, double c, double z,
                                                H2Plan* plan_out = nullptr) {
  H2Plan P = h2f1_plan(region, a, b, c, z);
  double g;
  if (P.method == kH2mSeries) {
    const H2Val sv = h2f1_direct<false>(P.p, P.q, c, P.x, kH2ConnTerms);
    g = sv.v;
    if (P.pfaff && !(sv.err <= 64.0 * kH2Ulp * fabs(sv.v))) {
      H2Plan Q = P;
      h2f1_set_swap(Q, a, b, c, !P.swap);
      const H2Val qv = h2f1_direct<false>(Q.p, Q.q, c, Q.x, kH2ConnTerms);
      if (qv.err / fabs(qv.v) < sv.err / fabs(sv.v)) {
        g = qv.v;
        P = Q;
      }
    }
  } else {
    const H2Val cv = h2f1_connect<false>(P.p, P.q, c, 1.0 - P.x);
    g = cv.v;
    if (!(cv.err <= 64.0 * kH2Ulp * fabs(cv.v))) {
      double best = isfinite(cv.v) ? cv.err / fabs(cv.v) : CUDART_INF;
      const H2Plan P0 = P;
      for (int k = 0; k < (P0.pfaff ? 2 : 1); ++k) {
        H2Plan Q = P0;
        if (k == 1) h2f1_set_swap(Q, a, b, c, !P0.swap);
        const H2Val dv = h2f1_direct<false>(Q.p, Q.q, c, Q.x, kH2DirectTerms);
        const double rel = dv.err / fabs(dv.v);
        if (rel < best) {
          best = rel;
          g = dv.v;
          P = Q;
          P.method = kH2mDirect;
        }
      }
      const double sg = c - P0.p - P0.q;
      if (!(best <= 1e-12) && fabs(sg - rint(sg)) < 1e-5) {
        const H2Val hv = h2f1_connect_shifted<false>(P0.p, P0.q, c, 1.0 - P0.x);
        if (hv.err / fabs(hv.v) < best) {
          g = hv.v;
          P = P0;
          P.method = kH2mShifted;
        }
      }
    }
  }
  if (plan_out) *plan_out = P;
  return P.pfaff ? exp(-P.p * P.lz) * g : g;
}

static __device__ __noinline__ double h2f1_value(double a, double b, double c, double z,
                                                 double eps = kH2f1Eps) {
  double v;
  if (h2f1_special(a, b, c, z, v, eps)) return v;
  return h2f1_eval(h2f1_region_of(z), a, b, c, z);
}

struct H2f1Grad {
  double v, da, db, dc, dz;
};

// F and its gradient from G(p, q; c; x) and G's derivatives, for a plan.
// Pfaff: F = (1-z)^-p G, x = z/(z-1), p = a, q = c - b (or p = b, q = c - a);
// dF/dz = p F/(1-z) - (1-z)^-p G'(x)/(1-z)^2.
__device__ inline H2f1Grad h2f1_assemble(const H2Plan& P, const H2Val& G, double z) {
  H2f1Grad g;
  if (!P.pfaff) {
    g.v = G.v;
    g.da = G.dp;
    g.db = G.dq;
    g.dc = G.dc;
    g.dz = G.dx;
    return g;
  }
  const double pre = exp(-P.p * P.lz), omz = 1.0 - z;
  g.v = pre * G.v;
  const double Fp = pre * (G.dp - P.lz * G.v), Fq = pre * G.dq;
  g.dc = pre * (G.dq + G.dc);
  if (!P.swap) {
    g.da = Fp;
    g.db = -Fq;
  } else {
    g.db = Fp;
    g.da = -Fq;
  }
  g.dz = P.p / omz * g.v - pre * G.dx / (omz * omz);
  return g;
}

// Value and derivatives by the evaluator and Pfaff variant of a plan (the
// plan's p, q are recomputed from a, b, c; x and lz depend on z only).
static __device__ __noinline__ H2f1Grad h2f1_param_grad(const H2Plan& plan, double a, double b, double c, double z) {
  H2Plan P = plan;
  if (P.pfaff) {
    h2f1_set_swap(P, a, b, c, plan.swap);
  } else {
    P.p = a;
    P.q = b;
  }
  return h2f1_assemble(P, h2f1_core<true>(P.method, P.p, P.q, c, P.x), z);
}

__device__ inline double h2f1_dz(double a, double b, double c, double z, double eps = kH2f1Eps) {
  return (a * b / c) * h2f1_value(a + 1.0, b + 1.0, c + 1.0, z, eps);
}

// Difference step in c: F has poles at c = 0, -1, -2, ..., so the step is
// also kept below 1/16 of the distance to the nearest one.
__device__ inline double h2f1_c_step(double c, double rel) {
  double h = rel * fmax(1.0, fabs(c));
  if (c < 0.5) h = fmin(h, fabs(c - rint(c)) * 0.0625);
  return h;
}

// Central differences of the value in (a, b, c), for the special points
// (the reference's own treatment outside its series region).
__device__ inline void h2f1_fd_grad(double a, double b, double c, double z, H2f1Grad& g, double eps = kH2f1Eps) {
  const double e3 = 6.0554544523933395e-06;  // ε^(1/3)
  const double ha = e3 * fmax(1.0, fabs(a)), hb = e3 * fmax(1.0, fabs(b)), hc = h2f1_c_step(c, e3);
  g.da = (h2f1_value(a + ha, b, c, z, eps) - h2f1_value(a - ha, b, c, z, eps)) / (2.0 * ha);
  g.db = (h2f1_value(a, b + hb, c, z, eps) - h2f1_value(a, b - hb, c, z, eps)) / (2.0 * hb);
  g.dc = (h2f1_value(a, b, c + hc, z, eps) - h2f1_value(a, b, c - hc, z, eps)) / (2.0 * hc);
}

// Full gradient (∂/∂a, ∂/∂b, ∂/∂c, ∂/∂z), with the region and plan used.
// Away from the special points it takes one evaluation with derivatives
// whenever the first evaluator is accurate (the common case); otherwise the
// evaluator is chosen as for the value (h2f1_eval) and evaluated again.
static __device__ __noinline__ H2f1Grad h2f1_grad(double a, double b, double c, double z, double eps = kH2f1Eps,
                                                  int* region_out = nullptr, H2Plan* plan_out = nullptr) {
  H2f1Grad g;
  double sv;
  if (h2f1_special(a, b, c, z, sv, eps)) {
    g.v = sv;
    g.dz = h2f1_dz(a, b, c, z, eps);
    h2f1_fd_grad(a, b, c, z, g, eps);
    if (region_out) *region_out = kH2Special;
    return g;
  }
  const int region = h2f1_region_of(z);
  H2Plan P = h2f1_plan(region, a, b, c, z);
  H2Val G;
  bool ok;
  if (P.method == kH2mSeries) {
    G = h2f1_direct<true>(P.p, P.q, c, P.x, kH2ConnTerms);
    if (P.pfaff && !(G.err <= 64.0 * kH2Ulp * fabs(G.v))) {
      H2Plan Q = P;
      h2f1_set_swap(Q, a, b, c, !P.swap);
      const H2Val GQ = h2f1_direct<true>(Q.p, Q.q, c, Q.x, kH2ConnTerms);
      if (GQ.err / fabs(GQ.v) < G.err / fabs(G.v)) {
        G = GQ;
        P = Q;
      }
    }
    ok = true;
  } else {
    G = h2f1_connect<true>(P.p, P.q, c, 1.0 - P.x);
    ok = G.err <= 64.0 * kH2Ulp * fabs(G.v);
  }
  if (!ok) {
    h2f1_eval(region, a, b, c, z, &P);
    G = h2f1_core<true>(P.method, P.p, P.q, c, P.x);
  }
  g = h2f1_assemble(P, G, z);
  if (region_out) *region_out = region;
  if (plan_out) *plan_out = P;
  return g;
}

// The two halves of h2f1_grad for the map kernel's rescue list.  The first
// returns false (g untouched) where h2f1_grad would fall back from the
// connection formula to the evaluator search; the second is that fallback
// alone.  Together they give h2f1_grad's results bit for bit, but the
// declined elements run their long series in full warps.
static __device__ __noinline__ bool h2f1_grad_first(double a, double b, double c, double z, double eps,
                                                    H2f1Grad& g) {
  double sv;
  if (h2f1_special(a, b, c, z, sv, eps)) {
    g.v = sv;
    g.dz = h2f1_dz(a, b, c, z, eps);
    h2f1_fd_grad(a, b, c, z, g, eps);
    return true;
  }
  const int region = h2f1_region_of(z);
  const H2Plan P = h2f1_plan(region, a, b, c, z);
  if (P.method == kH2mSeries) {
    g = h2f1_grad(a, b, c, z, eps);
    return true;
  }
  const H2Val G = h2f1_connect<true>(P.p, P.q, c, 1.0 - P.x);
  if (!(G.err <= 64.0 * kH2Ulp * fabs(G.v))) return false;
  g = h2f1_assemble(P, G, z);
  return true;
}
static __device__ __noinline__ H2f1Grad h2f1_grad_fallback(double a, double b, double c, double z) {
  H2Plan P;
  h2f1_eval(h2f1_region_of(z), a, b, c, z, &P);
  return h2f1_assemble(P, h2f1_core<true>(P.method, P.p, P.q, c, P.x), z);
}

// Hessian of F in (a, b, c, z), symmetric, packed as
// [aa, ab, ac, az, bb, bc, bz, cc, cz, zz], with the gradient.
struct H2f1Hess {
  H2f1Grad g;
  double h[10];
};
__device__ inline H2f1Hess h2f1_hessian(double a, double b, double c, double z, double eps = kH2f1Eps) {
  H2f1Hess H;
  int region = kH2Special;
  H2Plan plan;
  H.g = h2f1_grad(a, b, c, z, eps, &region, &plan);
  // z row from the gradient of F1 = F(a+1, b+1; c+1; z): ∂F/∂z = (ab/c) F1.
  const double k = a * b / c;
  const H2f1Grad g1 = h2f1_grad(a + 1.0, b + 1.0, c + 1.0, z, eps);
  H.h[3] = (b / c) * g1.v + k * g1.da;
  H.h[6] = (a / c) * g1.v + k * g1.db;
  H.h[8] = -(k / c) * g1.v + k * g1.dc;
  H.h[9] = k * g1.dz;
  double J[3][3];
  if (region == kH2Special) {
    // Second differences of the value, step ε^(1/4) max(1, |p|).
    const double e4 = 1.2207031250000000e-04;
    const double hs[3] = {e4 * fmax(1.0, fabs(a)), e4 * fmax(1.0, fabs(b)), h2f1_c_step(c, e4)};
    const double f0 = H.g.v;
    for (int i = 0; i < 3; ++i) {
      for (int j = i; j < 3; ++j) {
        double pp[3] = {a, b, c}, pm[3] = {a, b, c}, mp[3] = {a, b, c}, mm[3] = {a, b, c};
        if (i == j) {
          pp[i] += hs[i];
          mm[i] -= hs[i];
          J[i][i] = (h2f1_value(pp[0], pp[1], pp[2], z, eps) - 2.0 * f0 + h2f1_value(mm[0], mm[1], mm[2], z, eps)) /
                    (hs[i] * hs[i]);
        } else {
          pp[i] += hs[i], pp[j] += hs[j];
          pm[i] += hs[i], pm[j] -= hs[j];
          mp[i] -= hs[i], mp[j] += hs[j];
          mm[i] -= hs[i], mm[j] -= hs[j];
          J[i][j] = J[j][i] = (h2f1_value(pp[0], pp[1], pp[2], z, eps) - h2f1_value(pm[0], pm[1], pm[2], z, eps) -
                               h2f1_value(mp[0], mp[1], mp[2], z, eps) + h2f1_value(mm[0], mm[1], mm[2], z, eps)) /
                              (4.0 * hs[i] * hs[j]);
        }
      }
    }
  } else {
    // Central differences of the analytic gradient at steps h and 2h,
    // Richardson-extrapolated (error O(h^4)), evaluator held fixed;
    // h = ε^(1/5) max(1, |p|).  For c < 1/2 the differences are taken of the
    // gradient of F/Γ(c), which is entire in c, and the poles of Γ(c) are
    // put back analytically (ψ(c), ψ'(c)).
    const bool regc = c < 0.5;
    const double e5 = 7.4009597974140505e-04;
    const double hs[3] = {e5 * fmax(1.0, fabs(a)), e5 * fmax(1.0, fabs(b)), e5 * fmax(1.0, fabs(c))};
    for (int i = 0; i < 3; ++i) {
      double d1[3], d2[3];
      for (int m = 1; m <= 2; ++m) {
        double pa[3] = {a, b, c}, ma[3] = {a, b, c};
        pa[i] += m * hs[i];
        ma[i] -= m * hs[i];
        H2f1Grad gp = h2f1_param_grad(plan, pa[0], pa[1], pa[2], z);
        H2f1Grad gm = h2f1_param_grad(plan, ma[0], ma[1], ma[2], z);
        if (regc) {
          const double rp = rgamma_d(pa[2]), rm = rgamma_d(ma[2]);
          gp.dc = rp * (gp.dc - digamma_d(pa[2]) * gp.v);
          gp.da *= rp;
          gp.db *= rp;
          gm.dc = rm * (gm.dc - digamma_d(ma[2]) * gm.v);
          gm.da *= rm;
          gm.db *= rm;
        }
        const double inv = 1.0 / (2.0 * m * hs[i]);
        double* d = m == 1 ? d1 : d2;
        d[0] = (gp.da - gm.da) * inv;
        d[1] = (gp.db - gm.db) * inv;
        d[2] = (gp.dc - gm.dc) * inv;
      }
      for (int j = 0; j < 3; ++j) J[i][j] = (4.0 * d1[j] - d2[j]) / 3.0;
    }
    if (regc) {
      // F = Γ(c) F~: F_xy = Γ F~_xy (x, y in a, b); F_xc = ψ F_x + Γ F~_xc;
      // F_cc = (ψ' - ψ²) F + 2ψ F_c + Γ F~_cc.
      const double gc = tgamma(c), psi = digamma_d(c), psi1 = trigamma_d(c);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) J[i][j] *= gc;
      J[0][2] += psi * H.g.da;
      J[2][0] += psi * H.g.da;
      J[1][2] += psi * H.g.db;
      J[2][1] += psi * H.g.db;
      J[2][2] += (psi1 - psi * psi) * H.g.v + 2.0 * psi * H.g.dc;
    }
  }
  H.h[0] = J[0][0];
  H.h[1] = 0.5 * (J[0][1] + J[1][0]);
  H.h[2] = 0.5 * (J[0][2] + J[2][0]);
  H.h[4] = J[1][1];
  H.h[5] = 0.5 * (J[1][2] + J[2][1]);
  H.h[7] = J[2][2];
  return H;
}

}  // namespace tsb
