"""Device-driven batches (TMX_BATCH_GRAPH): the order loop and its block
rounds as one CUDA graph of conditional nodes that the GPU runs by itself.

The graph mode runs the same kernels on the same tables as the host-driven
loop, only scheduled by the device, so every result must equal the host
mode's bit for bit: final orders, status bits, the six per-grain sums, every
T-matrix and the gradients (which reuse the LU factors the graph's rounds
kept). Covered: the bench distribution (orders up to 32, every size bucket
up to 17..32 members), repeated batches on one context (the graph is built
once per batch shape and reused) and a batch after another one of other
grains (nothing may depend on what an earlier batch left in the buffers),
and a low maximum_order at which most grains stop unconverged at the last
order (the loop's exit with grains still in flight and the final round
after it).
"""
import numpy as np
import pytest

import _helpers as H
import oracle as O
from costuum_b200.tmatrix import Context, tmatrix_size

pytestmark = pytest.mark.gpu

SCHEDULE = dict(min_order=10, max_order=100, gauss_legendre_factor=2,
                tolerance=1e-4)


def _run(mode, r, lam, m, d, sched, reps=1, before=None):
    c = Context(0)
    try:
        c.set_batch_mode(mode)
        if before is not None:
            # another batch first: the compared one must not depend on what
            # an earlier batch left in the context's buffers
            c.tmatrix_batch(*before, **sched)
        out = []
        for _ in range(reps):
            res = c.tmatrix_batch(r, lam, m, d, **sched)
            flat, off = c.tmatrices()
            T = [flat[off[i]:off[i] + tmatrix_size(int(res.nmax[i]))].copy()
                 if res.nmax[i] > 0 else None for i in range(res.n)]
            out.append(dict(nmax=res.nmax.copy(), status=res.status.copy(),
                            q=res.q.copy(), T=T, mode=c.last_batch_mode))
        return out
    finally:
        c.close()


def _same(a, b):
    assert np.array_equal(a["nmax"], b["nmax"])
    assert np.array_equal(a["status"], b["status"])
    assert np.array_equal(a["q"], b["q"])
    for i, (x, y) in enumerate(zip(a["T"], b["T"])):
        assert (x is None) == (y is None), i
        if x is not None:
            assert np.array_equal(x, y), i


def test_graph_equals_host_bench_distribution():
    r, lam, m, d = H.config2_sample(2048, 31)
    host = _run(Context.BATCH_HOST, r, lam, m, d, SCHEDULE)[0]
    graph = _run(Context.BATCH_GRAPH, r, lam, m, d, SCHEDULE, reps=3)
    assert host["mode"] == Context.BATCH_HOST
    for g in graph:
        assert g["mode"] == Context.BATCH_GRAPH
        _same(g, host)
    assert (host["status"] == 0).all()


def test_graph_after_other_batches_equals_host():
    r, lam, m, d = H.config2_sample(1024, 34)
    other = H.config2_sample(1500, 35)
    host = _run(Context.BATCH_HOST, r, lam, m, d, SCHEDULE)[0]
    graph = _run(Context.BATCH_GRAPH, r, lam, m, d, SCHEDULE, reps=2, before=other)
    for g in graph:
        assert g["mode"] == Context.BATCH_GRAPH
        _same(g, host)


def test_graph_equals_host_unconverged_at_last_order():
    r, lam, m, d = H.config2_sample(700, 32)
    sched = dict(SCHEDULE, max_order=14)
    host = _run(Context.BATCH_HOST, r, lam, m, d, sched)[0]
    graph = _run(Context.BATCH_GRAPH, r, lam, m, d, sched)[0]
    assert graph["mode"] == Context.BATCH_GRAPH
    _same(graph, host)
    # most grains of x up to 10 do not converge below order 14
    assert (host["nmax"] == 13).sum() > 100


def test_graph_gradients_equal_host():
    r, lam, m, d = H.config2_sample(400, 33)
    th = np.array([0.4, 1.3, 2.5])
    co = O.orientation_coefficients(2, 0.5, 120)
    out = {}
    for mode in (Context.BATCH_HOST, Context.BATCH_GRAPH):
        c = Context(0)
        try:
            c.set_batch_mode(mode)
            c.tmatrix_batch(r, lam, m, d, **SCHEDULE)
            assert c.last_batch_mode == mode
            q = c.observables(th, co)
            out[mode] = (q, c.gradients(th, co))
        finally:
            c.close()
    (qh, (q2h, dqh)), (qg, (q2g, dqg)) = out[Context.BATCH_HOST], out[Context.BATCH_GRAPH]
    assert np.array_equal(qh, qg) and np.array_equal(q2h, q2g)
    assert np.array_equal(dqh, dqg)


def test_graph_extent_from_previous_batch():
    """The graph's orders end a margin above the previous batch's largest
    final order (and never shrink for the same schedule). A batch that needs
    more orders than that is computed again in the host-driven mode (same
    results), and the next graph covers it."""
    small = H.config2_sample(300, 36, xmin=0.1, xmax=1.0)   # orders ~10-12
    large = H.config2_sample(600, 37, xmin=5.0, xmax=10.0)  # orders up to ~32
    host = _run(Context.BATCH_HOST, *large, SCHEDULE)[0]
    c = Context(0)
    try:
        # the first batch (host-driven) sets the extent of the first graph
        c.tmatrix_batch(*small, **SCHEDULE)
        c.set_batch_mode(Context.BATCH_GRAPH)
        modes = []
        for _ in range(2):
            res = c.tmatrix_batch(*large, **SCHEDULE)
            flat, off = c.tmatrices()
            got = dict(nmax=res.nmax.copy(), status=res.status.copy(), q=res.q.copy(),
                       T=[flat[off[i]:off[i] + tmatrix_size(int(res.nmax[i]))].copy()
                          if res.nmax[i] > 0 else None for i in range(res.n)])
            _same(got, host)
            modes.append(c.last_batch_mode)
    finally:
        c.close()
    assert int(host["nmax"].max()) > 12 + 8
    assert modes == [Context.BATCH_HOST, Context.BATCH_GRAPH]


def test_graph_few_grains_per_call():
    """Calls of one to five grains (groups of eight orders from the first
    step, fewer slots than the group layout's 32 per order): every call
    equals the host-driven result, and all run as one graph (its extent only
    grows within the schedule)."""
    c = Context(0)
    modes = []
    try:
        for i, k in enumerate((1, 3, 5, 2, 1)):
            g = H.config2_sample(k, 60 + i)
            host = _run(Context.BATCH_HOST, *g, SCHEDULE)[0]
            c.set_batch_mode(Context.BATCH_GRAPH)
            res = c.tmatrix_batch(*g, **SCHEDULE)
            flat, off = c.tmatrices()
            got = dict(nmax=res.nmax.copy(), status=res.status.copy(), q=res.q.copy(),
                       T=[flat[off[j]:off[j] + tmatrix_size(int(res.nmax[j]))].copy()
                          if res.nmax[j] > 0 else None for j in range(res.n)])
            _same(got, host)
            modes.append(c.last_batch_mode)
    finally:
        c.close()
    assert modes.count(Context.BATCH_GRAPH) >= 3
