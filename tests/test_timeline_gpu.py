"""Launch timeline of a profiled batch (tmx_profile_timeline).

A batch computed with the profile on leaves one record per block and table
launch and three marks: the batch's start, the end of the order loop and the
end of the batch. The records must be ordered in time as the work flow
orders them (every launch inside the batch, the order loop's launches on the
library stream before the loop's end mark, block launches with work items),
the per-kernel sums of the timeline must equal tmx_profile_read's, and
switching the profile on again must clear the timeline.
"""
import ctypes

import numpy as np
import pytest

import _helpers as H
from costuum_b200 import _lib
from costuum_b200.tmatrix import Context

pytestmark = pytest.mark.gpu

SCHEDULE = dict(min_order=10, max_order=100, gauss_legendre_factor=2,
                tolerance=1e-4)


def test_timeline_of_a_batch(ctx):
    r, lam, m, d = H.config2_sample(600, 11)
    ctx.tmatrix_batch(r, lam, m, d, **SCHEDULE)
    ctx.profile(True)
    ctx.tmatrix_batch(r, lam, m, d, **SCHEDULE)
    tl = ctx.timeline()
    lib = _lib.load()
    sums = []
    for k in (0, 1):
        ms = np.zeros(1)
        n = ctypes.c_int64()
        rc = lib.tmx_profile_read(ctx._h, k, _lib.ptr(ms), ctypes.byref(n),
                                  _lib.ptr(np.zeros(1)))
        assert rc == 0
        sums.append((float(ms[0]), n.value))
    ctx.profile(False)

    marks = {int(k): float(s) for k, s in zip(tl["kind"], tl["start_ms"])
             if k < 0}
    assert set(marks) == {-1, -2, -3}
    t_start, t_loop, t_end = marks[-1], marks[-2], marks[-3]
    assert 0.0 <= t_start <= t_loop <= t_end
    runs = tl[tl["kind"] >= 0]
    assert np.all(runs["start_ms"] <= runs["end_ms"])
    assert np.all(runs["start_ms"] >= t_start - 1e-3)
    assert np.all(runs["end_ms"] <= t_end + 1e-3)
    assert set(runs["stream"].tolist()) <= set(range(9))
    blocks = runs[runs["kind"] == 0]
    assert blocks.size > 0 and np.all(blocks["items"] > 0)
    # the order loop runs on the library stream and ends before its mark
    loop = runs[runs["stream"] == 0]
    assert loop.size > 0 and loop["start_ms"].min() <= t_loop
    # same launches and (to float rounding of the event times) the same
    # per-kernel time as the profile counters
    for k, (ms, n) in enumerate(sums):
        sel = runs[runs["kind"] == k]
        assert sel.size == n
        assert abs(float((sel["end_ms"] - sel["start_ms"]).sum()) - ms) \
            <= 1e-3 * max(1.0, ms)

    ctx.profile(True)
    assert ctx.timeline().size == 0
    ctx.profile(False)


def test_host_times_of_a_batch(ctx):
    r, lam, m, d = H.config2_sample(600, 12)
    ctx.tmatrix_batch(r, lam, m, d, **SCHEDULE)
    ht = np.zeros(4)
    assert _lib.load().tmx_batch_host_times(ctx._h, _lib.ptr(ht)) == 0
    wall, blocked, setup, groups = ht
    assert wall > 0 and 0 <= blocked <= wall and 0 <= setup <= wall
    assert groups >= 1 and groups == int(groups)
