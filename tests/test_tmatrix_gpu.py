"""GPU parity of the batched T-matrix path against the CPU oracle.

Tolerances (the stated parity bounds): T-matrix elements 1e-9 relative in norm
(per m block, Frobenius), Q_ext 1e-8 relative.
"""
import numpy as np
import pytest

import oracle as O
import _helpers as H
from costuum_b200 import tmatrix as TM

pytestmark = pytest.mark.gpu

T_TOL = 1e-9
Q_TOL = 1e-8


def _compare(res, i, ref, nmax):
    assert res.nmax[i] == ref["nmax"], (i, res.nmax[i], ref["nmax"])
    Tg = res.tmatrix(i)
    worst = 0.0
    for m in range(nmax + 1):
        a = TM.block(Tg, nmax, m)
        b = O.block(ref["T"], nmax, m)
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        worst = max(worst, err)
    assert worst <= T_TOL, (i, worst)
    qref = ref["info"]
    for j in (0, 1, 2, 3):
        assert abs(res.q[i, j] - qref[j]) <= Q_TOL * abs(qref[j]), (i, j, res.q[i, j], qref[j])
    return worst


def test_config1_grain(ctx):
    # oblate d=2, r_ev 0.2 um, lambda 1 um, m = 1.5 + 0.02i, TaskManager schedule
    res = ctx.tmatrix_batch([0.2e-6], 1e-6, 1.5 + 0.02j, 2.0)
    ref = O.tmatrix_converge(0.2e-6, 1e-6, 1.5 + 0.02j, 2.0)
    assert res.status[0] == 0
    assert res.ngauss[0] == ref["ngauss"] == 2 * ref["nmax"]
    _compare(res, 0, ref, ref["nmax"])


@pytest.mark.parametrize("seed,xmax", [(7, 6.0), (11, 10.0)])
def test_config2_sample(ctx, seed, xmax):
    r, lam, m, d = H.config2_sample(24, seed, xmax=xmax)
    res = ctx.tmatrix_batch(r, lam, m, d, max_order=60)
    worst = 0.0
    differ = 0
    for i in range(len(r)):
        ref = O.tmatrix_converge(r[i], lam, m[i], d[i], max_order=60)
        err, diff = H.check_grain(res, i, r[i], lam, m[i], d[i], ref)
        worst = max(worst, err)
        differ += diff
    print("worst T rel err %.3g, %d rounding-regime nmax differences" % (worst, differ))
    assert differ <= len(r) // 4


def test_not_converged_and_bad_input(ctx):
    # max_order 12: the chain stops at order 11 without converging for x = 6
    r = np.array([6.0e-6 / (2 * np.pi), -1.0, 0.3e-6])
    res = ctx.tmatrix_batch(r, 1e-6, 1.4 + 0.01j, 1.5, max_order=12)
    assert res.status[0] & TM.GRAIN_NOT_CONVERGED
    assert res.nmax[0] == 11
    assert res.status[1] == TM.GRAIN_BAD_INPUT and res.nmax[1] == 0
    ref = O.tmatrix_converge(r[0], 1e-6, 1.4 + 0.01j, 1.5, max_order=12)
    assert not ref["converged"]
    _compare(res, 0, ref, 11)
    ref2 = O.tmatrix_converge(r[2], 1e-6, 1.4 + 0.01j, 1.5, max_order=12)
    _compare(res, 2, ref2, ref2["nmax"])


def test_empty_batch(ctx):
    res = ctx.tmatrix_batch(np.zeros(0), 1e-6, 1.5, 1.0)
    assert res.n == 0


def test_kernels_launched(ctx):
    before = ctx.kernel_launches
    ctx.tmatrix_batch([0.1e-6], 1e-6, 1.5 + 0.1j, 0.8)
    assert ctx.kernel_launches > before


def test_bessel_start_automatic_equals_800(ctx):
    """The automatic recurrence start gives the same T-matrices, bit for bit,
    as the reference's fixed start at n = 800."""
    r, lam, m, d = H.config2_sample(16, 5, xmax=10.0)
    a = ctx.tmatrix_batch(r, lam, m, d, max_order=50, bessel_start=0)
    Ta = [a.tmatrix(i) for i in range(len(r))]
    na = a.nmax.copy()
    b = ctx.tmatrix_batch(r, lam, m, d, max_order=50, bessel_start=800)
    assert np.array_equal(na, b.nmax)
    for i in range(len(r)):
        assert np.array_equal(Ta[i], b.tmatrix(i)), i


def test_two_block_rounds_match_one_round(ctx):
    # 1024 grains: most converge early, so the blocks of the converged grains
    # run while the order loop continues (two rounds on two streams); the
    # same blocks in one round (fixed orders) must give the same doubles
    r, lam, m, d = H.config2_sample(1024, 5)
    res = ctx.tmatrix_batch(r, lam, m, d)
    nm, ng, q = res.nmax.copy(), res.ngauss.copy(), res.q.copy()
    T2 = [res.tmatrix(i) for i in range(0, 1024, 7)]
    assert (res.status == 0).all()
    fix = ctx.tmatrix_batch_fixed(r, lam, m, d, nm, ng)
    assert np.array_equal(fix.q[:, 2:4], q[:, 2:4])
    for k, i in enumerate(range(0, 1024, 7)):
        assert np.array_equal(fix.tmatrix(i), T2[k]), i


def test_gradients_after_two_rounds(ctx):
    # gradients right after a two-round batch equal those after a fixed batch
    r, lam, m, d = H.config2_sample(1024, 6)
    th = np.array([0.3, 1.1, 2.0])
    res = ctx.tmatrix_batch(r, lam, m, d)
    nm, ng = res.nmax.copy(), res.ngauss.copy()
    q1, dq1 = ctx.gradients(th)
    ctx.tmatrix_batch_fixed(r, lam, m, d, nm, ng)
    q2, dq2 = ctx.gradients(th)
    assert np.array_equal(q1, q2)
    assert np.array_equal(dq1, dq2)
