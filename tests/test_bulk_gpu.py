"""Bulk T-matrix download, streamed T-matrices, and block rounds on a cold
context.

* tmx_batch_tmatrices returns every T-matrix of a batch in one transfer, at
  offsets that give the same matrices as the per-grain download;
* with a page-locked stream buffer the block rounds copy their ranges while
  the batch runs; the result must equal the plain download, also when the
  buffer holds only part of the batch (the rest is copied afterwards) and
  after the buffer has held another batch;
* a fresh context whose block rounds start at orders it has never seen grows
  its Wigner and quadrature tables while earlier rounds still run on the
  round streams; the T-matrices must equal, bit for bit, those of one round
  at the same orders (the fixed-order path) on another fresh context.
"""
import numpy as np
import pytest

import _helpers as H
from costuum_b200.tmatrix import Context

pytestmark = pytest.mark.gpu

SCHEDULE = dict(min_order=10, max_order=100, gauss_legendre_factor=2,
                tolerance=1e-4)


def _per_grain(res):
    return [res.tmatrix(i) for i in range(res.n)]


def test_bulk_download_equals_per_grain(ctx):
    r, lam, m, d = H.config2_sample(300, 7)
    res = ctx.tmatrix_batch(r, lam, m, d, **SCHEDULE)
    want = _per_grain(res)
    flat, off = ctx.tmatrices()
    for i in range(res.n):
        assert off[i] >= 0
        got = flat[off[i]:off[i] + want[i].size]
        assert np.array_equal(got, want[i]), i


def test_streamed_tmatrices(ctx):
    r, lam, m, d = H.config2_sample(1200, 8)
    res = ctx.tmatrix_batch(r, lam, m, d, **SCHEDULE)
    want = _per_grain(res)
    flat0, off0 = ctx.tmatrices()
    total = flat0.size
    try:
        # whole batch streamed; then a buffer that holds only a part
        for cap in (total + 1000, total // 3):
            ctx.stream_tmatrices(cap)
            # a different batch first, so the buffer holds stale data
            r2, lam2, m2, d2 = H.config2_sample(200, 9)
            ctx.tmatrix_batch(r2, lam2, m2, d2, **SCHEDULE)
            ctx.tmatrices()
            res = ctx.tmatrix_batch(r, lam, m, d, **SCHEDULE)
            flat, off = ctx.tmatrices()
            # (the layout follows the order in which grains became final,
            # which the convergence kernel's atomics may change from batch to
            # batch; each grain's matrix does not change)
            assert (off >= 0).all()
            for i in range(res.n):
                got = flat[off[i]:off[i] + want[i].size]
                assert np.array_equal(got, want[i]), (cap, i)
    finally:
        ctx.stream_tmatrices(0)


def test_rounds_on_cold_context_same_doubles():
    # grains that converge over a wide range of orders, so that several
    # rounds start at orders the fresh context has no tables for yet
    r, lam, m, d = H.config2_sample(2048, 11, xmin=0.1, xmax=10.0)
    a = Context(0)
    try:
        res = a.tmatrix_batch(r, lam, m, d, **SCHEDULE)
        assert (res.status == 0).all()
        got = _per_grain(res)
        nm, ng = res.nmax.copy(), res.ngauss.copy()
    finally:
        a.close()
    assert len(set(nm.tolist())) > 10
    b = Context(0)
    try:
        fix = b.tmatrix_batch_fixed(r, lam, m, d, nm, ng)
        for i in range(len(r)):
            assert np.array_equal(fix.tmatrix(i), got[i]), i
    finally:
        b.close()
