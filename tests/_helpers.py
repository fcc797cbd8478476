"""Shared helpers for the parity tests (test infrastructure)."""
import numpy as np

import oracle as O
from costuum_b200 import tmatrix as TM

T_TOL = 1e-9   # T-matrix: relative error of each m block in Frobenius norm
Q_TOL = 1e-8   # Qext / Qsca: relative error
ROUNDING = 1e-12  # relative Q change that only rounding can produce


def config2_sample(n, seed, xmin=0.1, xmax=10.0):
    """Seeded grains with the config-2 distributions (lambda = 1 um)."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(xmin, xmax, n)
    d = np.exp(rng.uniform(np.log(0.5), np.log(2.0), n))
    mr = rng.uniform(1.3, 2.0, n)
    mi = np.exp(rng.uniform(np.log(1e-3), np.log(1.0), n))
    lam = 1e-6
    r = x * lam / (2 * np.pi)
    return r, lam, mr + 1j * mi, d


def oracle_at(r, lam, m, d, nmax, ngauss):
    """Oracle T-matrix and m = 0 sums at a given (nmax, ngauss)."""
    T = np.zeros(O.tmatrix_size(nmax), np.complex128)
    T0, qs, qe = O.tmatrix_m0(r, lam, m, d, nmax, ngauss)
    T[:4 * nmax * nmax] = T0.ravel()
    for mm in range(1, nmax + 1):
        blk = O.tmatrix_mblock(r, lam, m, d, nmax, ngauss, mm)
        off = O.block_offset(nmax, mm)
        T[off:off + blk.size] = blk.ravel()
    fqs, fqe = O.tmatrix_q(T, nmax)
    return T, np.array([qs, qe, fqs, fqe])


def t_error(Ta, Tb, nmax):
    worst = 0.0
    for m in range(nmax + 1):
        a = TM.block(Ta, nmax, m)
        b = O.block(Tb, nmax, m)
        worst = max(worst, np.linalg.norm(a - b) / np.linalg.norm(b))
    return worst


def oracle_sensitivity(r, lam, m, d, nmax, ngauss, T, q, rel=1e-15):
    """The oracle's own change when r_ev moves by +-rel (a few ulps): the
    worst per-m-block relative change of T and the worst relative change of
    the four sums. For an ill-conditioned grain this is the part of any
    difference between two correct implementations that rounding alone
    produces."""
    t_s, q_s = 0.0, 0.0
    for f in (1 + rel, 1 - rel):
        T2, q2 = oracle_at(r * f, lam, m, d, nmax, ngauss)
        t_s = max(t_s, t_error(T2, T, nmax))
        q_s = max(q_s, max(abs(q2[j] - q[j]) / abs(q[j]) for j in range(4)))
    return t_s, q_s


def oracle_z181(r, lam, m, d, nmax, ngauss, coeffs):
    """The oracle's random-orientation (coeffs) scattering matrices for
    incidence along the axis at the 181 scattering angles 0..180 deg."""
    T, _ = oracle_at(r, lam, m, d, nmax, ngauss)
    Ta = O.orientation_average(T, nmax, coeffs[:2 * nmax + 1])
    tout = np.radians(np.arange(181.0))
    return np.stack([O.z_from_s(O.amplitude_lab(Ta, nmax, lam, 0., 0., 0., 0., t, 0.))
                     for t in tout])


def z_sensitivity(r, lam, m, d, nmax, ngauss, coeffs, rel=1e-15):
    """The oracle's own change of those 181 matrices (relative to each
    matrix's largest element) when r_ev moves by +-rel."""
    z0 = oracle_z181(r, lam, m, d, nmax, ngauss, coeffs)
    scale = np.max(np.abs(z0), axis=(-1, -2))
    s = 0.0
    for f in (1 + rel, 1 - rel):
        z = oracle_z181(r * f, lam, m, d, nmax, ngauss, coeffs)
        s = max(s, float(np.max(np.max(np.abs(z - z0), axis=(-1, -2)) / scale)))
    return s


def calculator_decision_band(r, lam, m, d, nmax, ndgs=2, tol=1e-4, rel=1e-15):
    """For the calculator's order test between orders nmax - 1 and nmax
    (ngauss = ndgs order): the oracle's change d = max(dQsca, dQext) and the
    rounding noise of the m = 0 sums (their relative change when r_ev moves
    by +-rel). Returns (|d - tol|, noise): a decision with |d - tol| within
    a few times the noise is set by rounding."""
    def sums(rr, k):
        return np.array(O.tmatrix_m0(rr, lam, m, d, k, ndgs * k)[1:])
    qa, qb = sums(r, nmax - 1), sums(r, nmax)
    dq = np.max(np.abs((qa - qb) / qb))
    noise = 0.0
    for f in (1 + rel, 1 - rel):
        for k, q0 in ((nmax - 1, qa), (nmax, qb)):
            noise = max(noise, float(np.max(np.abs((sums(r * f, k) - q0) / q0))))
    return abs(dq - tol), noise


def check_grain(res, i, r, lam, m, d, ref):
    """Compare grain i of a GPU batch with the oracle's convergence run.

    The converged order must agree unless the oracle's own change between
    orders is at rounding level (the reference's test is dQ > 0 and
    dQ <= tolerance, so bitwise-equal sums of consecutive orders delay its
    convergence by an amount that depends only on rounding). T and the sums
    are compared at the GPU's (nmax, ngauss)."""
    N = int(res.nmax[i])
    if N != ref["nmax"]:
        lo = min(N, ref["nmax"])
        hi = max(N, ref["nmax"])
        qs = [O.tmatrix_m0(r, lam, m, d, k, res.ngauss[i] // N * k)[1:]
              for k in range(lo - 1, hi + 1)]
        for a, b in zip(qs[:-1], qs[1:]):
            for j in (0, 1):
                assert abs(a[j] - b[j]) <= ROUNDING * abs(b[j]), (
                    "converged order differs outside the rounding regime",
                    i, N, ref["nmax"])
    T, q = oracle_at(r, lam, m, d, N, int(res.ngauss[i]))
    err = t_error(res.tmatrix(i), T, N)
    assert err <= T_TOL, (i, err)
    for j in range(4):
        assert abs(res.q[i, j] - q[j]) <= Q_TOL * abs(q[j]), (i, j, res.q[i, j], q[j])
    return err, N != ref["nmax"]
