"""The plain path (CosTuuM.TMatrix: calculator schedule, orientation
average, K and Z at one orientation, absorption cross sections).

CPU: the oracle's restatement (oracle/tmx_oracle.c) against the reference
module's own outputs (tests/golden/plain.npz, made by make_golden.py) and a
few rows of the reference's Mishchenko-code fixture
(test/test_tmatrixcalculator.txt, stored as the array mish_rows).
GPU: the library against the same fixtures, all 101 fixture rows in one
batch, and the oracle.

Tolerances: orders exact; K, Z and cross sections of the library within 1e-8
of the largest element of each matrix (the T-matrices agree to ~1e-12, the
orientation average and the amplitude sums are reassociated); the
Mishchenko fixture at the reference test's own bounds (Q 1e-5, Z 2e-2,
relative to |a + b| as in test/Assert.hpp; testTMatrixCalculator.cpp:111-132).
"""
import os

import numpy as np
import pytest

import oracle as O

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MAT_TOL = 1e-8


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(G, "plain.npz"))


def _case(gold, i):
    r, d, lam, mr, mi, c2b, ev = gold["plain_args"][i]
    r_ev = r if ev else O.rv_over_rs(d) * r
    return r_ev, d, lam, complex(mr, mi), c2b


def _coeffs(c2b, d, nmax):
    order = 2 * nmax
    if c2b in (0.0, 1.0):
        return O.orientation_coefficients(2, d, order)
    if c2b == 1.0 / 3.0:
        return O.orientation_coefficients(0, 0.0, order)
    return O.orientation_coefficients(1, c2b, order)


def _oracle_tmatrix(r_ev, d, lam, m, c2b):
    nmax, ngauss, st = O.calculator_orders(r_ev, lam, m, d)
    assert st == 0
    T = O.full_tmatrix(r_ev, lam, m, d, nmax, ngauss)
    if c2b >= 0:
        T = O.orientation_average(T, nmax, _coeffs(c2b, d, nmax))
    return nmax, ngauss, T


def _close(a, b, tol=MAT_TOL):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.max(np.abs(b))
    return np.max(np.abs(a - b)) <= tol * scale, np.max(np.abs(a - b)) / scale


def _rel_ok(a, b, tol):
    """The reference test's relative check (test/Assert.hpp:67-72):
    |a - b| <= tol |a + b|."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= tol * np.abs(a + b))


def _mish(row):
    """Inputs of one fixture row in SI units (testTMatrixCalculator.cpp:64-108)."""
    axi, rat, lam, mrr, mri, eps, ddelt, ndgs = row[:8]
    alpha, beta, thet0, thet, phi0, phi = np.radians(row[8:14])
    axi *= 1e-6
    lam *= 1e-6
    ratio = O.rv_over_rs(eps) if abs(rat - 1.0) > 1e-8 else 1.0
    return dict(r_ev=ratio * axi, lam=lam, m=complex(mrr, mri), d=eps,
                tol=0.1 * ddelt, ndgs=int(ndgs), angles=(alpha, beta, thet0, phi0,
                                                        thet, phi),
                qsca=row[14], qext=row[15], walb=row[16],
                Z=row[17:33].reshape(4, 4) * 1e-12)


# ------------------------------------------------------------------- CPU ---

@pytest.mark.parametrize("i", [0, 1, 2, 3])
def test_oracle_plain_against_reference(gold, i):
    r_ev, d, lam, m, c2b = _case(gold, i)
    nmax, _, T = _oracle_tmatrix(r_ev, d, lam, m, c2b)
    assert nmax == int(gold["p%d_nmax" % i][0])
    th, ph = [0.3, 1.2], [0.0, 0.7]
    for a in range(2):
        for b in range(2):
            S = O.amplitude_lab(T, nmax, lam, 0.4, 0.9, th[a], ph[b], th[a], ph[b])
            ok, err = _close(O.k_from_s(lam, S), gold["p%d_K" % i][a, b], 1e-12)
            assert ok, (i, a, b, err)
    S = O.amplitude_lab(T, nmax, lam, 0.3, 1.1, 0.5, 0.1, 1.7, 2.2)
    ok, err = _close(O.z_from_s(S), gold["p%d_Z" % i], 1e-12)
    assert ok, (i, err)


def test_oracle_mishchenko_rows(gold):
    rows = gold["mish_rows"]
    for row in rows[[0, 3, 17, 40, 77]]:
        c = _mish(row)
        nmax, ngauss, st = O.calculator_orders(c["r_ev"], c["lam"], c["m"], c["d"],
                                               200, c["tol"], c["ndgs"], 500)
        assert st == 0
        T = O.full_tmatrix(c["r_ev"], c["lam"], c["m"], c["d"], nmax, ngauss)
        qsca, qext = O.tmatrix_q(T, nmax)
        assert _rel_ok(qext, c["qext"], 1e-5)
        assert _rel_ok(qsca, c["qsca"], 1e-5)
        assert _rel_ok(-qsca / qext, c["walb"], 1e-5)
        Z = O.z_from_s(O.amplitude_lab(T, nmax, c["lam"], *c["angles"]))
        assert _rel_ok(Z, c["Z"], 2e-2), (Z, c["Z"])


# ------------------------------------------------------------------- GPU ---

@pytest.mark.gpu
@pytest.mark.parametrize("i", [0, 1, 2, 3, 4])
def test_tmatrix_class_against_reference(gold, i):
    from costuum_b200 import CosTuuM as C
    r, d, lam, mr, mi, c2b, ev = gold["plain_args"][i]
    T = C.TMatrix(r, d, lam, complex(mr, mi), cos2beta=c2b,
                  is_equal_volume_radius=bool(ev))
    assert T.get_nmax() == int(gold["p%d_nmax" % i][0])
    K = T.get_extinction_matrix(np.array([0.3, 1.2]), np.array([0.0, 0.7]),
                                alpha=0.4, beta=0.9)
    for a in range(2):
        for b in range(2):
            ok, err = _close(K[a, b], gold["p%d_K" % i][a, b])
            assert ok, (i, a, b, err)
    Z = T.get_scattering_matrix(0.5, 0.1, 1.7, 2.2, alpha=0.3, beta=1.1)
    ok, err = _close(Z, gold["p%d_Z" % i])
    assert ok, (i, err)
    if i < 4:
        cabs = T.get_absorption_cross_sections(np.array([0.4, 1.3]), ngauss=10)
        ok, err = _close(cabs, gold["p%d_cabs" % i])
        assert ok, (i, err)
        c1 = T.get_absorption_cross_section(np.array([0.4, 1.3]), ngauss=10)
        assert np.allclose(c1, cabs[:, 0], rtol=0, atol=1e-30)
        avg = T.get_average_absorption_cross_section()
        assert abs(avg - gold["p%d_avg" % i][0]) <= MAT_TOL * abs(gold["p%d_avg" % i][0])
    else:
        z181 = T.get_scattering_matrix(0.0, 0.0, np.radians(np.arange(181.0)), 0.0)
        for j in range(181):
            ok, err = _close(z181[j], gold["p4_z181"][j])
            assert ok, (j, err)


@pytest.mark.gpu
def test_mishchenko_fixture_all_rows(ctx, gold):
    rows = gold["mish_rows"]
    cs = [_mish(r) for r in rows]
    # rows share tol and ndgs per run: group them
    keys = sorted({(c["tol"], c["ndgs"]) for c in cs})
    n_checked = 0
    for tol, ndgs in keys:
        sel = [j for j, c in enumerate(cs) if c["tol"] == tol and c["ndgs"] == ndgs]
        res = ctx.tmatrix_batch_calculator(
            [cs[j]["r_ev"] for j in sel], [cs[j]["lam"] for j in sel],
            [cs[j]["m"] for j in sel], [cs[j]["d"] for j in sel],
            maximum_order=200, tolerance=tol, gauss_legendre_factor=ndgs,
            maximum_ngauss=500)
        assert (res.status == 0).all(), res.status
        ang = np.array([cs[j]["angles"] for j in sel])
        Z = ctx.scattering_matrix(np.arange(len(sel)), ang[:, 2], ang[:, 3],
                                  ang[:, 4], ang[:, 5], ang[:, 0], ang[:, 1])
        for q, j in enumerate(sel):
            c = cs[j]
            qsca, qext = res.qsca[q], res.qext[q]
            assert _rel_ok(qext, c["qext"], 1e-5), (j, qext, c["qext"])
            assert _rel_ok(qsca, c["qsca"], 1e-5), (j, qsca, c["qsca"])
            assert _rel_ok(-qsca / qext, c["walb"], 1e-5), j
            assert _rel_ok(Z[q], c["Z"], 2e-2), j
            n_checked += 1
    assert n_checked == len(rows)


@pytest.mark.gpu
def test_calculator_orders_match_oracle(ctx):
    rng = np.random.default_rng(3)
    n = 12
    x = rng.uniform(0.5, 12.0, n)
    d = np.exp(rng.uniform(np.log(0.5), np.log(2.0), n))
    m = rng.uniform(1.3, 1.8, n) + 1j * np.exp(rng.uniform(np.log(1e-3), 0.0, n))
    lam = 1e-6
    r = x * lam / (2 * np.pi)
    res = ctx.tmatrix_batch_calculator(r, lam, m, d)
    for i in range(n):
        nmax, ngauss, st = O.calculator_orders(r[i], lam, m[i], d[i])
        assert res.status[i] == st
        assert (res.nmax[i], res.ngauss[i]) == (nmax, ngauss), i
        T = O.full_tmatrix(r[i], lam, m[i], d[i], nmax, ngauss)
        Tg = res.tmatrix(i)
        assert np.linalg.norm(Tg - T) <= 1e-9 * np.linalg.norm(T), i


@pytest.mark.gpu
def test_orientation_average_matches_oracle(ctx):
    r, lam, m, d = [0.25e-6, 0.4e-6], 1e-6, [1.5 + 0.02j, 1.6 + 0.3j], [0.7, 1.8]
    res = ctx.tmatrix_batch_calculator(r, lam, m, d)
    T = [res.tmatrix(i) for i in range(2)]
    nm = [int(v) for v in res.nmax]
    top = 2 * max(nm)
    sets = np.stack([O.orientation_coefficients(1, 0.6, top),
                     O.orientation_coefficients(2, 0.5, top)])
    ctx.orientation_average(sets, [0, 1])
    for i in range(2):
        Ta = O.orientation_average(T[i], nm[i], sets[i][:2 * nm[i] + 1])
        Tg = res.tmatrix(i)
        assert np.linalg.norm(Tg - Ta) <= 1e-10 * np.linalg.norm(Ta), i
    with pytest.raises(Exception):
        ctx.gradients([0.5])
