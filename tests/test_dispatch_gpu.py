"""Block-kernel dispatch table and its autotuner (tmx_get_dispatch,
tmx_set_dispatch, tmx_autotune).

Every kernel family is run in every size bucket it can serve, on two grains
at fixed orders whose parity classes cover all five buckets (order 40:
classes of 1..40 members; order 70: up to 70), and compared with the oracle
(T within 1e-9 relative per m block, or 4x the oracle's own change under a
1e-15 change of r_ev where that is larger; the full-T sums within 1e-8).
The autotuner must time each family in each bucket it can serve, move a
bucket only to the fastest family and only when it beats the current one by
5 %, and leave results that still match the oracle.
"""
import numpy as np
import pytest

import _helpers as H

pytestmark = pytest.mark.gpu

LAM = 1e-6
X = np.array([12.0, 24.0])
R_EV = X * LAM / (2 * np.pi)
M = np.array([1.5 + 0.01j, 1.5 + 0.01j])
D = np.array([1.4, 0.8])
NMAX = np.array([40, 70], np.int32)
NGAUSS = 2 * NMAX
CAPACITY = (8, 16, 32, 64, 128)
TOP = (8, 16, 32, 64, 128)
DEFAULT = [0, 1, 2, 3, 4]


@pytest.fixture(scope="module")
def refs():
    out = []
    for i in range(len(X)):
        args = (R_EV[i], LAM, M[i], D[i], int(NMAX[i]), int(NGAUSS[i]))
        T, q = H.oracle_at(*args)
        t_s, q_s = H.oracle_sensitivity(*args, T, q)
        out.append((T, q, max(H.T_TOL, 4 * t_s), max(H.Q_TOL, 4 * q_s)))
    return out


def _check(res, refs):
    assert (res.status == 0).all(), res.status
    for i, (T, q, t_tol, q_tol) in enumerate(refs):
        err = H.t_error(res.tmatrix(i), T, int(NMAX[i]))
        assert err <= t_tol, (i, err)
        # the full-T sums (the fixed-order path has no m = 0 chain sums)
        for j in (2, 3):
            assert abs(res.q[i, j] - q[j]) <= q_tol * abs(q[j]), (i, j)


def test_default_table(ctx):
    assert list(ctx.get_dispatch()) == DEFAULT


def test_set_dispatch_rejects_a_family_too_small(ctx):
    with pytest.raises(Exception):
        ctx.set_dispatch([0, 0, 2, 3, 4])  # DFMA tiles hold 8 members, not 16
    with pytest.raises(Exception):
        ctx.set_dispatch([0, 1, 2, 3, 7])
    assert list(ctx.get_dispatch()) == DEFAULT


@pytest.mark.parametrize("family", range(5))
def test_family_in_every_bucket_it_serves(ctx, refs, family):
    table = [family if CAPACITY[family] >= TOP[b] else DEFAULT[b] for b in range(5)]
    ctx.set_dispatch(table)
    try:
        assert list(ctx.get_dispatch()) == table
        _check(ctx.tmatrix_batch_fixed(R_EV, LAM, M, D, NMAX, NGAUSS), refs)
    finally:
        ctx.set_dispatch(DEFAULT)


def test_autotune(ctx, refs):
    try:
        table, ms = ctx.autotune(R_EV, LAM, M, D, NMAX, NGAUSS, reps=2)
        print("tuned table", list(table))
        print(np.array2string(ms, precision=4))
        for b in range(5):
            for f in range(5):
                if CAPACITY[f] >= TOP[b]:
                    assert ms[b, f] > 0, (b, f)
                else:
                    assert ms[b, f] == -1, (b, f)
            # the fastest family, when at least 5 % faster than the default
            best = min(ms[b, f] for f in range(5) if ms[b, f] > 0)
            if table[b] != DEFAULT[b]:
                assert ms[b, table[b]] == best, b
                assert best < 0.95 * ms[b, DEFAULT[b]], b
            else:
                assert best >= 0.95 * ms[b, DEFAULT[b]], b
        _check(ctx.tmatrix_batch_fixed(R_EV, LAM, M, D, NMAX, NGAUSS), refs)
    finally:
        ctx.set_dispatch(DEFAULT)
