"""The CPU oracle (oracle/tmx_oracle.c) against the reference's own outputs.

The fixtures in tests/golden/ were produced by the unmodified reference
(tests/golden/make_golden.py). The restatement keeps the reference's
operation order, so the comparisons are exact.
"""
import os

import numpy as np
import pytest

import oracle as O

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def stages():
    return np.load(os.path.join(G, "stages.npz"))


@pytest.fixture(scope="module")
def tms():
    return np.load(os.path.join(G, "tmatrices.npz"))


def test_gauss_legendre(stages):
    for order in (1, 2, 3, 5, 20, 41, 80):
        x, w = O.gauss_legendre(order)
        assert np.array_equal(x, stages["gl_%d_x" % order])
        assert np.array_equal(w, stages["gl_%d_w" % order])


def test_gauss_legendre_closed_forms():
    # testSpecialFunctions.cpp: n = 1..5 against closed forms (1e-7 there)
    x, w = O.gauss_legendre(2)
    assert np.allclose(x, [-1 / np.sqrt(3), 1 / np.sqrt(3)], atol=1e-15)
    assert np.allclose(w, [1, 1], atol=1e-15)
    x, w = O.gauss_legendre(3)
    assert np.allclose(x, [-np.sqrt(0.6), 0, np.sqrt(0.6)], atol=1e-15)
    assert np.allclose(w, [5 / 9, 8 / 9, 5 / 9], atol=1e-15)


def test_bessel(stages):
    for i in range(4):
        z = stages["bj_%d_z" % i][0]
        j, dj = O.bessel_j_real(30, z)
        y, dy = O.bessel_y_real(30, z)
        assert np.array_equal(np.stack([j, dj, y, dy]), stages["bj_%d" % i])
    for i in range(3):
        z = stages["bjc_%d_z" % i][0]
        j, dj = O.bessel_j_complex(30, z)
        assert np.array_equal(np.stack([j, dj]), stages["bjc_%d" % i])


def test_wigner(stages):
    for i in range(4):
        c, m = stages["wig_%d_arg" % i]
        d, dd = O.wigner_d(c, 20, int(m))
        assert np.array_equal(np.stack([d, dd]), stages["wig_%d" % i])


def test_clebsch_gordan(stages):
    for i in range(4):
        n1, n2, N = (int(v) for v in stages["cg_%d_arg" % i])
        assert np.array_equal(O.clebsch_gordan_row(n1, n2, N), stages["cg_%d" % i])
    # known value: <1 0 1 0 | 0 0> = -1/sqrt(3)
    assert abs(O.clebsch_gordan_row(1, 1, 0)[1] + 1 / np.sqrt(3)) < 1e-15


def test_orientation_coefficients(stages):
    for i in range(4):
        kind, par = stages["od_%d_arg" % i]
        assert np.array_equal(O.orientation_coefficients(int(kind), par, 20),
                              stages["od_%d" % i])


def test_plu_inverse(stages):
    assert np.array_equal(O.plu_inverse(stages["plu_a"]), stages["plu_inv"])


def test_rv_over_rs(stages):
    got = np.array([O.rv_over_rs(d) for d in (0.5, 2.0, 1.0, 3.3)])
    assert np.array_equal(got, stages["rvrs"])
    # testSpecialFunctions.cpp known values (rel 1e-10)
    assert abs(got[0] / 0.9637112829756893 - 1) < 1e-10
    assert abs(got[1] / 0.955443263377723 - 1) < 1e-10


def test_tmatrix_chain(tms):
    grains = tms["t_grains"]
    for i, (r, lam, mr, mi, d) in enumerate(grains):
        res = O.tmatrix_converge(r, lam, mr + 1j * mi, d, max_order=40)
        nmax, ngauss, conv = tms["t_%d_meta" % i]
        assert res["nmax"] == nmax and res["ngauss"] == ngauss
        assert res["converged"] == bool(conv)
        assert np.array_equal(res["T"], tms["t_%d_T" % i])
        assert np.array_equal(res["info"], tms["t_%d_q" % i])


def test_get_table_one_grain():
    """The one-grain configuration through the oracle's observables equals the
    reference module's get_table output bit for bit."""
    tab = np.load(os.path.join(G, "tables.npz"))
    th = tab["gt1_theta"]
    res = O.tmatrix_converge(0.2e-6, 1e-6, 1.5 + 0.02j, 2.0, max_order=40)
    N = res["nmax"]
    coeffs = O.orientation_coefficients(0, 0., 80)  # random: r < minimum size
    Ta = O.orientation_average(res["T"], N, coeffs)
    ab = O.absorption(Ta, N, 1e-6, 0.2e-6, th)
    ex = O.extinction(Ta, N, 1e-6, 0.2e-6, th)
    assert np.array_equal(np.concatenate([ab, ex], axis=1), tab["gt1"])
    assert abs(tab["gt1"][0, 0] - 0.515661805) < 1e-9
