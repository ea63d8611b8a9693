"""The oracle pinned before it is trusted: the C restatement against the
reference's own outputs (golden fixtures made from the reference's compiled
scalar kernels) and against the known-answer tests in the reference's test
suite; the reference's accuracy bands against scipy/mpmath."""

import math

import numpy as np
import pytest

from oracle import oracle as O
from tests._util import golden, rel_err, ulp_err


@pytest.mark.parametrize("name", ["log_gamma", "gamma", "digamma", "trigamma"])
def test_restatement_matches_reference_outputs_gamma_family(name):
    d = golden("gamma_family")
    x = d["x"]
    m = x > 0  # the reference's real recurrences are the restated ones for x > 0
    got = O.restated(name, 0, x[m])[0]
    assert ulp_err(got, d[f"ref_{name}"][m]).max() <= 2
    if name != "gamma":
        got = O.restated(name, 1, d["g"][m], x[m])[0]
        assert ulp_err(got, d[f"ref_{name}_backward"][m]).max() <= 2


@pytest.mark.parametrize("name,key", [("regularized_gamma_p", "p"), ("regularized_gamma_q", "q")])
def test_restatement_matches_reference_outputs_igamma(name, key):
    d = golden("igamma")
    got = O.restated(name, 0, d["a"], d["x"])[0]
    assert ulp_err(got, d[f"ref_{name}"]).max() <= 2
    ga, gx = O.restated(name, 1, d["g"], d["a"], d["x"])
    assert ulp_err(ga, d[f"ref_{name}_grad_a"]).max() <= 2
    assert ulp_err(gx, d[f"ref_{name}_grad_x"]).max() <= 2


@pytest.mark.parametrize("name,key", [("complete_legendre_elliptic_integral_k", "k"), ("complete_legendre_elliptic_integral_e", "e")])
def test_restatement_matches_reference_outputs_elliptic(name, key):
    d = golden("elliptic")
    got = O.restated(name, 0, d["m"])[0]
    assert ulp_err(got, d[f"ref_{key}"]).max() <= 2


def test_known_answers_from_reference_tests():
    # test__log_gamma.py:149-165 known values and half value
    z = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 0.5])
    want = np.array([0.0, 0.0, math.log(2), math.log(6), math.log(24), 0.5 * math.log(math.pi)])
    np.testing.assert_allclose(O.restated("log_gamma", 0, z)[0], want, rtol=1e-8, atol=1e-8)
    # test__log_gamma.py:178-183 recurrence lnΓ(z+1) = lnΓ(z) + ln z
    z = np.array([0.5, 1.5, 2.5, 5.0, 10.0])
    np.testing.assert_allclose(O.restated("log_gamma", 0, z + 1)[0], O.restated("log_gamma", 0, z)[0] + np.log(z), rtol=1e-10, atol=1e-10)
    # test__log_gamma.py:185-192 pole at 0
    assert np.isinf(O.restated("log_gamma", 0, np.array([0.0]))[0]).all()
    # test__regularized_gamma_p.py:30-56: P(a,0)=0, P(1,x)=1-e^-x, P(a,100)->1, range
    a = np.array([0.5, 1.0, 2.0, 10.0])
    assert np.all(O.restated("regularized_gamma_p", 0, a, 0 * a)[0] == 0)
    x = np.linspace(0.1, 5.0, 50)
    np.testing.assert_allclose(O.restated("regularized_gamma_p", 0, np.ones_like(x), x)[0], 1 - np.exp(-x), atol=1e-6)
    np.testing.assert_allclose(O.restated("regularized_gamma_p", 0, np.array([1.0, 2.0, 5.0]), np.full(3, 100.0))[0], 1.0, atol=1e-10)
    rng = np.random.default_rng(0)
    p = O.restated("regularized_gamma_p", 0, rng.random(100) * 10 + 0.1, rng.random(100) * 20)[0]
    assert np.all((p >= 0) & (p <= 1))


def test_reference_accuracy_bands():
    """Where the reference is accurate (parity at 4 ulp + its own error is meaningful)
    and where it is not (graded against scipy/mpmath only)."""
    g = golden("gamma_family")
    x = g["x"]
    pos = x > 0
    zero_band = (np.abs(x - 1) < 0.1) | (np.abs(x - 2) < 0.1)
    e = rel_err(g["ref_log_gamma"], g["truth_log_gamma"])
    assert e[pos & ~zero_band].max() < 1e-13
    e = rel_err(g["ref_gamma"], g["truth_gamma"])
    assert e[pos & (x < 100)].max() < 1e-12
    # digamma: truncated 3-term asymptotic -> ~1e-8 (defect band)
    e = rel_err(g["ref_digamma"], g["truth_digamma"])
    assert 1e-10 < np.median(e[pos & (x < 5)])
    ig = golden("igamma")
    e = rel_err(ig["ref_regularized_gamma_p"], ig["truth_p"], floor=1e-280)
    assert np.nanmax(e[ig["truth_p"] > 1e-280]) < 1e-8
    el = golden("elliptic")
    m = el["m"]
    inside = (m >= 0) & (m < 1 - 1e-12)
    assert rel_err(el["ref_k"], el["truth_k"])[inside].max() < 1e-13
    # E(1) and m -> 1 are where the reference's R_G form loses accuracy
    assert rel_err(el["ref_e"], el["truth_e"])[inside].max() < 1e-12


def _same(x, y):
    return bool(np.all((x == y) | (np.isnan(x) & np.isnan(y))))


def test_restatement_matches_reference_outputs_hyp2f1():
    """The 2F1 restatement is bit-identical to the reference's compiled scalar
    kernel: forward on the benchmark sample and the special points, backward
    (analytic and finite-difference branches) on its first 300 points."""
    d = golden("hyp2f1")
    assert _same(O.restated("hypergeometric_2_f_1", 0, d["a"], d["b"], d["c"], d["z"])[0], d["ref"])
    sp = d["special"]
    assert _same(O.restated("hypergeometric_2_f_1", 0, *sp.T)[0], d["special_ref"])
    m = d["g"].size
    got = O.restated("hypergeometric_2_f_1", 1, d["g"], d["a"][:m], d["b"][:m], d["c"][:m], d["z"][:m], n_out=4)
    for k in range(4):
        assert _same(got[k], d["ref_grad"][:, k])


def test_hyp2f1_known_answers_from_reference_tests():
    """test__hypergeometric_2_f_1.py:2604-2703 (scipy values, tolerances as there)."""
    k = golden("hyp2f1")["kat"]
    got = O.restated("hypergeometric_2_f_1", 0, *k[:, :4].T)[0]
    fin = np.isfinite(k[:, 4])
    np.testing.assert_allclose(got[fin], k[fin, 4], rtol=1e-8, atol=1e-8)
    assert np.isposinf(got[~fin]).all()


def test_hyp2f1_reference_accuracy_bands():
    """The reference is accurate for z < 1/2 away from cancellation and wrong
    near z = 1, where its 2000-term series has not converged."""
    d = golden("hyp2f1")
    e = rel_err(d["ref"], d["truth"])
    z = d["z"]
    assert np.median(e[z < 0.5]) < 1e-14
    assert e[z >= 0.95].max() > 1e-3
    assert np.median(e[z >= 0.99]) > 1e-8


def test_incomplete_beta_fixture_pinned():
    """The incomplete_beta fixture: mpmath truth against scipy's betainc
    (an independent implementation) and the beta density, and the
    reference's own outputs stored beside them within the reference's
    accuracy (its fraction stops at 200 terms, so a, b >= 300 are left out)."""
    import scipy.special as sp
    import scipy.stats as st

    d = golden("incomplete_beta")
    x, a, b = d["x"], d["a"], d["b"]
    np.testing.assert_allclose(d["truth_v"], sp.betainc(a, b, x), rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(d["truth_dx"], st.beta.pdf(x, a, b), rtol=1e-10, atol=1e-300)
    small = (a < 300) & (b < 300)
    np.testing.assert_allclose(d["ref"][small], d["truth_v"][small], rtol=0, atol=1e-11)


def test_incomplete_beta_known_answers_from_reference_tests():
    """The reference's own known answers (incomplete_beta_test.cpp:70-114):
    I_z(1, 1) = z, I_z(1, b) = 1 - (1-z)^b, I_z(a, 1) = z^a and
    I_z(a, b) + I_(1-z)(b, a) = 1, checked on the stored mpmath truth's
    generator (scipy here) and on the reference's compiled kernel where built."""
    import scipy.special as sp

    from oracle import oracle as O

    z = np.array([0.1, 0.25, 0.5, 0.75, 0.9])
    np.testing.assert_allclose(sp.betainc(1.0, 3.0, z), 1 - (1 - z) ** 3, rtol=1e-13)
    np.testing.assert_allclose(sp.betainc(3.0, 1.0, z), z**3, rtol=1e-13)
    if not O.reference_available():
        pytest.skip("reference library not built")
    (u,) = O.reference("incomplete_beta", 0, np.array([0.0, 0.25, 0.5, 0.75, 1.0]), 1.0, 1.0)
    np.testing.assert_allclose(u, [0.0, 0.25, 0.5, 0.75, 1.0], atol=1e-12)
    (s1,) = O.reference("incomplete_beta", 0, z, 2.5, 3.5)
    (s2,) = O.reference("incomplete_beta", 0, 1 - z, 3.5, 2.5)
    np.testing.assert_allclose(s1 + s2, 1.0, atol=1e-10)
