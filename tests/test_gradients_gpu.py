"""Derivatives of orientation-averaged extinction coefficients with respect
to (Re m, Im m, r_ev, axis ratio): the tangent kernels against central finite
differences at the converged order, of the GPU forward and of the CPU oracle.
Tolerance 1e-6 relative (per grain, coefficient and parameter, over the
angles); 1e-5 for the large grains of test_tangents_large_grains, where the
differences themselves are no better.

A central difference has its own error: truncation O(h^2) for large steps,
rounding noise of the forward divided by h for small ones. For weakly
polarised grains (Qextpol ~ 1e-3 Qext) the noise floor of a 1e-6 relative
step is itself ~1e-6, so each derivative is compared with central
differences at relative steps 1e-6 and 1e-5 and the closer one must agree."""
import numpy as np
import pytest

import _helpers as H
import oracle as O

pytestmark = pytest.mark.gpu

FD_STEP = 1e-6
TOL = 1e-6


def _step(params, p):
    """Relative step: 1e-6 of r_ev and of d; for Re m and Im m 1e-6 of |m|
    (Im m can be 1e-3, where 1e-6 of it would put the forward's rounding
    noise at the 1e-6 level of the derivative)."""
    if p < 2:
        return FD_STEP * np.hypot(params[..., 0], params[..., 1])
    return FD_STEP * np.abs(params[..., p])
THETAS = np.array([0.3, 1.1, 1.9, 2.7])


def _coeffs(kind, param, order=120):
    return O.orientation_coefficients(kind, param, order)


def _fd_gpu(ctx, params, lam, nmax, ngauss, coeffs, rel=FD_STEP):
    n = len(params)
    fd = np.zeros((n, len(THETAS), 3, 4))
    for p in range(4):
        h = _step(params, p) * (rel / FD_STEP)
        out = []
        for sgn in (1, -1):
            q = params.copy()
            q[:, p] += sgn * h
            ctx.tmatrix_batch_fixed(q[:, 2], lam, q[:, 0] + 1j * q[:, 1], q[:, 3],
                                    nmax, ngauss)
            out.append(ctx.observables(THETAS, coeffs))
        fd[:, :, :, p] = (out[0] - out[1]) / (2 * h[:, None, None])
    return fd


def _compare(dq, fds, q, tol=TOL):
    """Relative error per (grain, coefficient, parameter). A coefficient that
    is zero up to rounding (Qextpol and Qextcpol under random orientation)
    has derivatives at the noise level of the same parameter's Qext
    derivative; there both must stay below 1e-6 of that scale."""
    worst = 0.0
    for i in range(dq.shape[0]):
        for p in range(4):
            scale = np.linalg.norm(dq[i, :, 0, p])
            for k in range(3):
                a = dq[i, :, k, p]
                errs = []
                for fd in fds:
                    b = fd[i, :, k, p]
                    nb = np.linalg.norm(b)
                    if nb < 1e-6 * scale:
                        # zero up to rounding: the tangent must be as well
                        errs.append(0.0 if np.linalg.norm(a) < 1e-6 * scale else 1.0)
                    else:
                        errs.append(np.linalg.norm(a - b) / nb)
                err = min(errs)
                worst = max(worst, err)
                assert err <= tol, (i, k, p, err)
    return worst


@pytest.mark.parametrize("kind,param", [(0, 0.0), (2, 2.0), (1, 0.3)])
def test_tangents_vs_central_differences(ctx, kind, param):
    r, lam, m, d = H.config2_sample(8, 17, xmax=6.0)
    params = np.stack([m.real, m.imag, r, d], axis=1)
    res = ctx.tmatrix_batch(r, lam, m, d, max_order=60)
    nmax, ngauss = res.nmax.copy(), res.ngauss.copy()
    coeffs = _coeffs(kind, param)
    ctx.tmatrix_batch_fixed(r, lam, m, d, nmax, ngauss)
    q, dq = ctx.gradients(THETAS, coeffs)
    assert np.allclose(q, ctx.observables(THETAS, coeffs), rtol=1e-12, atol=0)
    fds = [_fd_gpu(ctx, params, lam, nmax, ngauss, coeffs, rel)
           for rel in (1e-6, 1e-5)]
    worst = _compare(dq, fds, q)
    print("worst relative error vs central FD: %.3g" % worst)


def test_tangents_large_grains(ctx):
    """Grains of size parameter 16-35 (converged orders 29, 44, 52: classes
    beyond 32 members, the CTA tangent kernel) against central differences
    of the GPU forward at the converged orders. Bound 1e-5: for the x = 35
    grain the forward's Qext carries rounding noise of ~1e-11 relative (Q is
    ill-conditioned at order 52), so central differences resolve its
    derivatives to ~2e-6 at best (steps 1e-6 to 3e-5 relative), while the
    smaller grains agree to 1e-7."""
    lam = 1e-6
    x = np.array([16.0, 24.0, 35.0])
    r = x * lam / (2 * np.pi)
    m = np.array([1.5 + 0.05j, 1.4 + 0.01j, 1.6 + 0.1j])
    d = np.array([1.5, 0.7, 1.3])
    res = ctx.tmatrix_batch(r, lam, m, d, max_order=128)
    assert (res.status == 0).all(), res.status
    nmax, ngauss = res.nmax.copy(), res.ngauss.copy()
    assert nmax.max() > 32, nmax
    coeffs = _coeffs(0, 0.0, order=2 * int(nmax.max()))
    ctx.tmatrix_batch_fixed(r, lam, m, d, nmax, ngauss)
    q, dq = ctx.gradients(THETAS, coeffs)
    params = np.stack([m.real, m.imag, r, d], axis=1)
    fds = [_fd_gpu(ctx, params, lam, nmax, ngauss, coeffs, rel)
           for rel in (1e-6, 1e-5, 3e-5)]
    worst = _compare(dq, fds, q, tol=1e-5)
    print("large grains: nmax %s, worst relative error vs central FD: %.3g"
          % (list(nmax), worst))


def _oracle_q(r, lam, m, d, nmax, ngauss, coeffs):
    T, _ = H.oracle_at(r, lam, m, d, nmax, ngauss)
    Ta = O.orientation_average(T, nmax, coeffs)
    return O.extinction(Ta, nmax, lam, r, THETAS)


def test_tangents_vs_oracle_finite_differences(ctx):
    r, lam, m, d = H.config2_sample(3, 23, xmax=4.0)
    res = ctx.tmatrix_batch(r, lam, m, d, max_order=40)
    nmax, ngauss = res.nmax.copy(), res.ngauss.copy()
    coeffs = _coeffs(2, 0.5)
    ctx.tmatrix_batch_fixed(r, lam, m, d, nmax, ngauss)
    q, dq = ctx.gradients(THETAS, coeffs)
    params = np.stack([m.real, m.imag, r, d], axis=1)
    fds = []
    for rel in (1e-6, 1e-5):
        fd = np.zeros_like(dq)
        for i in range(3):
            for p in range(4):
                h = _step(params[i], p) * (rel / FD_STEP)
                vals = []
                for sgn in (1, -1):
                    x = params[i].copy()
                    x[p] += sgn * h
                    vals.append(_oracle_q(x[2], lam, x[0] + 1j * x[1], x[3],
                                          int(nmax[i]), int(ngauss[i]), coeffs))
                fd[i, :, :, p] = (vals[0] - vals[1]) / (2 * h)
        fds.append(fd)
    _compare(dq, fds, q)


def _oracle_fd_grain(job):
    """Central differences of the oracle's averaged extinction for one grain
    at its fixed order: (params, lam, nmax, ngauss, coeffs) -> fd[rel][theta,
    k, p] for the relative steps 1e-6 and 1e-5 (runs in a pool worker)."""
    params, lam, nmax, ngauss, coeffs = job
    out = []
    for rel in (1e-6, 1e-5):
        fd = np.zeros((len(THETAS), 3, 4))
        for p in range(4):
            h = _step(params, p) * (rel / FD_STEP)
            vals = []
            for sgn in (1, -1):
                x = params.copy()
                x[p] += sgn * h
                vals.append(_oracle_q(x[2], lam, x[0] + 1j * x[1], x[3], nmax,
                                      ngauss, coeffs))
            fd[:, :, p] = (vals[0] - vals[1]) / (2 * h)
        out.append(fd)
    return out


def test_tangents_vs_oracle_fd_64_grains(ctx, oracle_pool):
    """The seeded 64-grain subset of the 4096-grain batch (config-2
    distributions, seed 1; x in [0.1, 10], orders 10-32): tangents at the
    converged orders against central differences of the CPU oracle (the
    reference's algorithm, pinned bit for bit to it) at the same orders,
    within 1e-6."""
    r, lam, m, d = H.config2_sample(4096, 1)
    pick = np.sort(np.random.default_rng(64).choice(4096, 64, replace=False))
    r, m, d = r[pick], m[pick], d[pick]
    res = ctx.tmatrix_batch(r, lam, m, d, min_order=10, max_order=100)
    assert (res.status == 0).all()
    nmax, ngauss = res.nmax.copy(), res.ngauss.copy()
    coeffs = _coeffs(2, 0.5, order=2 * int(nmax.max()))
    q, dq = ctx.gradients(THETAS, coeffs)
    params = np.stack([m.real, m.imag, r, d], axis=1)
    jobs = [(params[i], lam, int(nmax[i]), int(ngauss[i]), coeffs)
            for i in range(len(r))]
    per = oracle_pool.map(_oracle_fd_grain, jobs)
    fds = [np.stack([p[k] for p in per]) for k in range(2)]
    worst = _compare(dq, fds, q)
    print("64 grains (orders %d-%d): worst relative error vs oracle FD %.3g"
          % (nmax.min(), nmax.max(), worst))


def test_autograd_function(ctx):
    import torch
    from costuum_b200.autograd import extinction
    r, lam, m, d = H.config2_sample(4, 29, xmax=5.0)
    coeffs = _coeffs(2, 2.0)
    params = torch.tensor(np.stack([m.real, m.imag, r, d], axis=1),
                          dtype=torch.float64, requires_grad=True)
    q = extinction(params, lam, THETAS, coeffs, max_order=50)
    w = torch.tensor(np.random.default_rng(0).standard_normal(q.shape))
    (q * w).sum().backward()
    res = ctx.tmatrix_batch(r, lam, m, d, max_order=50)
    ctx.tmatrix_batch_fixed(r, lam, m, d, res.nmax, res.ngauss)
    qq, dq = ctx.gradients(THETAS, coeffs)
    assert np.allclose(q.detach().numpy(), qq, rtol=1e-12)
    want = np.einsum("ntk,ntkp->np", w.numpy(), dq)
    assert np.allclose(params.grad.numpy(), want, rtol=1e-12, atol=0)


def test_autograd_backward_after_another_batch(ctx):
    """Backward right after its forward reuses the forward's LU factors;
    backward after another batch ran on the same context recomputes the
    blocks at the forward's orders. Both give the same gradient."""
    import torch
    from costuum_b200 import autograd as AG
    r, lam, m, d = H.config2_sample(6, 31, xmax=8.0)
    coeffs = _coeffs(0, 0.0)
    w = torch.tensor(np.random.default_rng(1).standard_normal((6, len(THETAS), 3)))
    grads = []
    for other in (False, True):
        params = torch.tensor(np.stack([m.real, m.imag, r, d], axis=1),
                              dtype=torch.float64, requires_grad=True)
        q = AG.extinction(params, lam, THETAS, coeffs, max_order=60)
        if other:
            r2, lam2, m2, d2 = H.config2_sample(5, 32)
            AG._context().tmatrix_batch(r2, lam2, m2, d2, max_order=60)
        (q * w).sum().backward()
        grads.append(params.grad.numpy().copy())
    assert np.allclose(grads[0], grads[1], rtol=1e-12, atol=0)


def test_observable_plan_reuse():
    """The observable plan (jobs, angles, coefficients on the device) that
    observables() builds is reused by the gradients of the same batch when
    the angles and coefficients are the same, and rebuilt when they or the
    batch differ: every call must give the doubles of a fresh context."""
    from costuum_b200.tmatrix import Context
    r, lam, m, d = H.config2_sample(300, 21)
    co_a = _coeffs(0, 0.0)
    co_b = _coeffs(2, 0.5)
    th_b = np.array([0.2, 0.9, 2.2])

    def fresh(thetas, coeffs):
        c = Context(0)
        try:
            c.tmatrix_batch(r, lam, m, d)
            return c.gradients(thetas, coeffs)
        finally:
            c.close()

    want_a = fresh(THETAS, co_a)
    want_b = fresh(th_b, co_b)
    ctx = Context(0)
    try:
        ctx.tmatrix_batch(r, lam, m, d)
        for thetas, coeffs, want in ((THETAS, co_a, want_a), (th_b, co_b, want_b),
                                     (THETAS, co_a, want_a)):
            q = ctx.observables(thetas, coeffs)
            assert np.array_equal(q, want[0])
            got = ctx.gradients(thetas, coeffs)  # the plan of observables()
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
        # angles changed between observables() and gradients()
        ctx.observables(THETAS, co_a)
        got = ctx.gradients(th_b, co_b)
        assert np.array_equal(got[1], want_b[1])
        # a new batch of other grains with the same angles and coefficients
        r2, lam2, m2, d2 = H.config2_sample(200, 22)
        ctx.tmatrix_batch(r2, lam2, m2, d2)
        c2 = Context(0)
        try:
            c2.tmatrix_batch(r2, lam2, m2, d2)
            want2 = c2.gradients(THETAS, co_a)
        finally:
            c2.close()
        got = ctx.gradients(THETAS, co_a)
        assert np.array_equal(got[1], want2[1])
    finally:
        ctx.close()


def test_gradients_reuse_forward_amplitudes():
    """After observables() on the same batch, angles and coefficients, the
    gradient pass takes the T-matrices' amplitudes from that call and runs
    the observable kernels on the three tangents only: q must then equal
    observables() exactly, and q and dq must agree with a gradient pass that
    computes all four (within 1e-12 of each coefficient's scale: the same
    arithmetic per matrix, in kernels compiled for three or four)."""
    from costuum_b200.tmatrix import Context
    r, lam, m, d = H.config2_sample(256, 41)
    co = _coeffs(2, 0.5)
    c = Context(0)
    try:
        c.tmatrix_batch(r, lam, m, d, min_order=10, max_order=100,
                        gauss_legendre_factor=2, tolerance=1e-4)
        q_all, dq_all = c.gradients(THETAS, co)
        q_all, dq_all = q_all.copy(), dq_all.copy()
        c.tmatrix_batch(r, lam, m, d, min_order=10, max_order=100,
                        gauss_legendre_factor=2, tolerance=1e-4)
        q_obs = c.observables(THETAS, co).copy()
        q_re, dq_re = c.gradients(THETAS, co)
    finally:
        c.close()
    assert np.array_equal(q_re, q_obs)
    scale_q = np.abs(q_all).max(axis=1, keepdims=True) + 1e-300
    assert (np.abs(q_re - q_all) <= 1e-12 * scale_q).all()
    scale = np.abs(dq_all).max(axis=(1, 2), keepdims=True) + 1e-300
    assert (np.abs(dq_re - dq_all) <= 1e-12 * scale).all()
