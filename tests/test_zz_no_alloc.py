"""The allocation-free entry point tmx_tmatrix_fixed_noalloc.

It serves callers that cannot allocate device memory (an application whose
device memory belongs to another framework's allocator, or a per-call path
that cannot afford cudaMalloc's implicit synchronisation); it keeps its
intermediates in a static device array shared by every call. This test calls
it through the C ABI and compares it with the batched entry point on calls
in a row (different grains back to back, so leftovers of one call in the
shared array must not leak into the next). The output buffer is filled with
NaN first, so every element must be written, and the device status word
starts at -1, so the call must report the grain's status bits (0 here).
"""
import ctypes

import numpy as np
import pytest

from costuum_b200 import _lib
from costuum_b200 import tmatrix as TM

pytestmark = pytest.mark.gpu

T_TOL = 1e-9


def _call(lib, g, nmax, ngauss, buf, stream, status=None):
    r, lam, m, d = g
    st = ctypes.c_void_p(status.data_ptr() if status is not None else None)
    return lib.tmx_tmatrix_fixed_noalloc(r, lam, m.real, m.imag, d, int(nmax),
                                         int(ngauss), ctypes.c_void_p(buf.data_ptr()),
                                         st, ctypes.c_void_p(stream))


def test_noalloc_matches_batch(ctx):
    import torch
    lib = _lib.load()
    grains = [(0.3e-6, 1e-6, 1.5 + 0.02j, 1.6), (0.6e-6, 1e-6, 1.8 + 0.2j, 0.7),
              (0.9e-6, 1e-6, 1.35 + 0.004j, 1.9)]
    res = ctx.tmatrix_batch([g[0] for g in grains], 1e-6, [g[2] for g in grains],
                            [g[3] for g in grains], max_order=33)
    stream = torch.cuda.current_stream().cuda_stream
    for i in (0, 1, 2, 0):  # calls in a row, each checked
        N, ng = int(res.nmax[i]), int(res.ngauss[i])
        assert N <= 32 and ng <= 64
        buf = torch.full((2 * TM.tmatrix_size(N),), float("nan"),
                         dtype=torch.float64, device="cuda")
        status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        rc = _call(lib, grains[i], N, ng, buf, stream, status)
        assert rc == 0
        torch.cuda.current_stream().synchronize()
        assert int(status.item()) == 0
        got = buf.cpu().numpy().view(np.complex128)
        want = res.tmatrix(i)
        for m in range(N + 1):
            a = TM.block(got, N, m)
            b = TM.block(want, N, m)
            assert np.all(np.isfinite(a))
            assert np.linalg.norm(a - b) <= T_TOL * np.linalg.norm(b), (i, m)


def test_noalloc_rejects_sizes_beyond_limit():
    import torch
    lib = _lib.load()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    g = (0.3e-6, 1e-6, 1.5 + 0.02j, 1.6)
    assert _call(lib, g, 33, 66, buf, 0) == -1
    assert _call(lib, g, 20, 65, buf, 0) == -1
