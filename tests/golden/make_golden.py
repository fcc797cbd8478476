"""Generate the golden fixtures in tests/golden/ from the unmodified reference.

Run in a container where the reference has been built (oracle/build_ref.sh),
with COSTUUM_REFERENCE naming the reference source tree (for its test data):
    COSTUUM_REFERENCE=<reference root> python tests/golden/make_golden.py \
        [stages tmatrices tables plain draine config5]
It imports the reference's own CPython module (oracle/_ref/CosTuuM*.so) and
its task objects (oracle/_ref/libref_driver.so) and stores their outputs.
The fixtures pin the C restatement in oracle/ (tests/test_oracle_golden.py).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("COSTUUM_REFERENCE", "")
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402
from oracle import _p  # noqa: E402


def stages():
    R = O.ref()
    out = {}
    for order in (1, 2, 3, 5, 20, 41, 80):
        x = np.zeros(order)
        w = np.zeros(order)
        R.ref_gauss_legendre(order, _p(x), _p(w))
        out["gl_%d_x" % order] = x
        out["gl_%d_w" % order] = w
    for i, z in enumerate((0.05, 1.3, 7.7, 33.1)):
        j = np.zeros(30)
        dj = np.zeros(30)
        y = np.zeros(30)
        dy = np.zeros(30)
        R.ref_bessel_j_real(30, z, _p(j), _p(dj))
        R.ref_bessel_y_real(30, z, _p(y), _p(dy))
        out["bj_%d" % i] = np.stack([j, dj, y, dy])
        out["bj_%d_z" % i] = np.array([z])
    for i, z in enumerate((0.3 + 0.01j, 2.5 + 0.3j, 12.0 + 1.5j)):
        j = np.zeros(30, complex)
        dj = np.zeros(30, complex)
        R.ref_bessel_j_complex(30, z.real, z.imag, _p(j), _p(dj))
        out["bjc_%d" % i] = np.stack([j, dj])
        out["bjc_%d_z" % i] = np.array([z])
    for i, (c, m) in enumerate(((-0.99, 0), (-0.3, 1), (0.1, 3), (0.9999, 10))):
        d = np.zeros(20)
        dd = np.zeros(20)
        R.ref_wigner_d(c, 20, m, _p(d), _p(dd))
        out["wig_%d" % i] = np.stack([d, dd])
        out["wig_%d_arg" % i] = np.array([c, m])
    for i, (n1, n2, N) in enumerate(((1, 1, 0), (3, 5, 4), (10, 7, 12), (20, 20, 40))):
        buf = np.zeros((N + 1) * (2 * n1 + 1))
        k = R.ref_clebsch_gordan_row(n1, n2, N, _p(buf))
        out["cg_%d" % i] = buf[:k].copy()
        out["cg_%d_arg" % i] = np.array([n1, n2, N])
    for i, (kind, par) in enumerate(((0, 0.), (1, 0.6), (2, 2.), (2, 0.5))):
        c = np.zeros(21)
        R.ref_orientation_coefficients(kind, par, 20, _p(c))
        out["od_%d" % i] = c
        out["od_%d_arg" % i] = np.array([kind, par])
    # random orientation at order 200 (the coefficients of maximum_order 100)
    c = np.zeros(201)
    R.ref_orientation_coefficients(0, 0., 200, _p(c))
    out["od_random_200"] = c
    A = (np.random.default_rng(0).standard_normal((7, 7))
         + 1j * np.random.default_rng(1).standard_normal((7, 7)))
    Ai = A.copy()
    R.ref_plu_inverse(7, _p(Ai))
    out["plu_a"] = A
    out["plu_inv"] = Ai
    out["rvrs"] = np.array([R.ref_rv_over_rs(d) for d in (0.5, 2.0, 1.0, 3.3)])
    c = np.zeros(41)
    R.ref_custom_orientation_coefficients(40, _p(c))
    out["od_custom"] = c  # p(beta) = 0.5 + 0.3 cos^2 beta
    for i, (n, cut, frac) in enumerate(((20, 0.15, -1.), (7, 0.3, -1.), (10, 0.15, 0.5))):
        sh = np.zeros(n)
        w = np.zeros(n)
        lim = np.zeros(2)
        R.ref_draine_hensley(n, cut, frac, _p(sh), _p(w), _p(lim))
        out["dh_%d" % i] = np.concatenate([sh, w, lim])
        out["dh_%d_arg" % i] = np.array([n, cut, frac])
    return out


GRAINS = [  # r_ev (m), wavelength (m), m, axis ratio
    (0.2e-6, 1e-6, 1.5 + 0.02j, 2.0),     # the one-grain configuration
    (0.5e-6, 1e-6, 1.7 + 0.1j, 0.6),
    (0.8e-6, 1e-6, 1.35 + 0.003j, 1.4),
    (0.05e-6, 1e-6, 1.9 + 0.8j, 0.9),
]


def tmatrices():
    out = {}
    r = [g[0] for g in GRAINS]
    lam = [g[1] for g in GRAINS]
    m = [g[2] for g in GRAINS]
    d = [g[3] for g in GRAINS]
    res = O.ref_batch(r, lam, m, d, max_order=40, nthreads=2)
    for i, rec in enumerate(res):
        out["t_%d_T" % i] = rec["T"]
        out["t_%d_meta" % i] = np.array([rec["nmax"], rec["ngauss"],
                                         int(rec["converged"])])
        out["t_%d_q" % i] = rec["q"]
    out["t_grains"] = np.array([[g[0], g[1], g[2].real, g[2].imag, g[3]]
                                for g in GRAINS])
    return out


def tables():
    """get_table outputs of the reference's Python module."""
    C = O.ref_module()
    out = {}
    th = np.arccos(np.linspace(-1, 1, 32))
    # the one-grain configuration: Q_ext / Q_abs at 32 zenith angles
    res = C.get_table(types=np.array([0]), sizes=np.array([0.2e-6]),
                      wavelengths=np.array([1e-6]), thetas=th,
                      shape_distribution=C.SingleShapeShapeDistribution(2.0),
                      alignment_distribution=C.SizeBasedAlignmentDistribution(
                          1e-5, C.DAVIS_GREENSTEIN_ALIGNMENT, maximum_order=40),
                      dust_properties=C.CustomDustProperties(lambda w, s, t: 1.5 + 0.02j),
                      number_of_threads=2, maximum_order=40, do_extinction=True)
    out["gt1"] = res
    out["gt1_theta"] = th
    # a small grid with alignment, Draine-Hensley shapes, scattering
    th2 = np.array([0.3, 1.2, 2.0])
    sizes = np.array([0.05e-6, 0.3e-6])
    lams = np.array([1.5e-6, 0.8e-6])
    mfun = lambda w, s, t: (1.4 + 0.3 * s / 1e-6) + 0.05j * (1e-6 / w)  # noqa: E731
    res2 = C.get_table(types=np.array([0]), sizes=sizes, wavelengths=lams,
                       thetas=th2,
                       shape_distribution=C.DraineHensleyShapeDistribution(4),
                       alignment_distribution=C.SizeBasedAlignmentDistribution(
                           0.1e-6, C.MISHCHENKO_ALIGNMENT, maximum_order=30),
                       dust_properties=C.CustomDustProperties(mfun),
                       number_of_threads=2, maximum_order=30,
                       do_extinction=True, do_scattering=True)
    out["gt2_qabs"] = res2[0]
    out["gt2_z"] = res2[1]
    out["gt2_theta"] = th2
    out["gt2_sizes"] = sizes
    out["gt2_lams"] = lams
    # scattering subtraction, Davis-Greenstein alignment, two compositions
    th3 = np.array([0.1, 1.0, 2.5])
    res3 = C.get_table(types=np.array([0, 2]), sizes=np.array([0.4e-6]),
                       wavelengths=np.array([1e-6, 2e-6]), thetas=th3,
                       shape_distribution=C.SingleShapeShapeDistribution(1.5),
                       alignment_distribution=C.SizeBasedAlignmentDistribution(
                           1e-7, C.DAVIS_GREENSTEIN_ALIGNMENT, maximum_order=30),
                       dust_properties=C.CustomDustProperties(
                           lambda w, s, t: (1.4 + 0.1 * t) + 0.05j),
                       number_of_threads=2, maximum_order=30,
                       number_of_quadrature_angles=6,
                       account_for_scattering=True)
    out["gt3"] = res3
    out["gt3_theta"] = th3
    # disabled alignment (prolate) and custom alignment (oblate/prolate)
    th4 = np.array([0.5, 1.5])
    res4 = C.get_table(types=np.array([0]), sizes=np.array([0.3e-6]),
                       wavelengths=np.array([1e-6]), thetas=th4,
                       shape_distribution=C.SingleShapeShapeDistribution(0.7),
                       alignment_distribution=C.SizeBasedAlignmentDistribution(
                           1e-7, C.DISABLE_ALIGNMENT, maximum_order=30),
                       dust_properties=C.CustomDustProperties(lambda w, s, t: 1.6 + 0.2j),
                       number_of_threads=2, maximum_order=30, do_extinction=True)
    out["gt4"] = res4
    out["gt4_theta"] = th4
    ob = C.MishchenkoOrientationDistribution(0.7, 60)
    pr = C.DavisGreensteinOrientationDistribution(0.5, 60)
    res5 = C.get_table(types=np.array([0]), sizes=np.array([0.3e-6]),
                       wavelengths=np.array([1e-6]), thetas=th4,
                       shape_distribution=C.SingleShapeShapeDistribution(0.7),
                       alignment_distribution=C.SizeBasedAlignmentDistribution(
                           1e-7, C.CUSTOM_ALIGNMENT, 30, ob, pr),
                       dust_properties=C.CustomDustProperties(lambda w, s, t: 1.6 + 0.2j),
                       number_of_threads=2, maximum_order=30, do_extinction=True)
    out["gt5"] = res5
    return out


# plain-path cases: (radius, axis ratio, wavelength, m, cos2beta,
# is_equal_volume_radius)
PLAIN = [
    (0.2e-6, 2.0, 1e-6, 1.5 + 0.02j, -1.0, True),
    (0.2e-6, 2.0, 1e-6, 1.5 + 0.02j, 1.0 / 3.0, True),
    (0.5e-6, 0.6, 1.2e-6, 1.7 + 0.1j, 0.6, False),
    (0.3e-6, 1.5, 0.9e-6, 1.4 + 0.05j, 1.0, True),
    (1.9e-6, 0.5, 1e-6, 1.5 + 0.02j, 1.0 / 3.0, True),
]


def plain():
    """Outputs of the reference module's TMatrix object (the plain path) and
    the Mishchenko-code fixture of the reference's calculator test."""
    C = O.ref_module()
    out = {}
    rows = []
    with open(os.path.join(REFERENCE, "test", "test_tmatrixcalculator.txt")) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            rows.append([float(v) for v in line.split()])
    out["mish_rows"] = np.array(rows)
    th = np.array([0.3, 1.2])
    ph = np.array([0.0, 0.7])
    for i, (r, d, lam, m, c2b, ev) in enumerate(PLAIN):
        T = C.TMatrix(r, d, lam, m, cos2beta=c2b, is_equal_volume_radius=ev)
        out["p%d_nmax" % i] = np.array([T.get_nmax()])
        out["p%d_K" % i] = T.get_extinction_matrix(th, ph, alpha=0.4, beta=0.9)
        out["p%d_Z" % i] = T.get_scattering_matrix(0.5, 0.1, 1.7, 2.2,
                                                   alpha=0.3, beta=1.1)
        if i < 4:
            out["p%d_cabs" % i] = T.get_absorption_cross_sections(
                np.array([0.4, 1.3]), ngauss=10)
            out["p%d_avg" % i] = np.array([T.get_average_absorption_cross_section()])
        if i == 4:
            tout = np.radians(np.arange(181.0))
            out["p4_z181"] = T.get_scattering_matrix(0.0, 0.0, tout, 0.0)
    out["plain_args"] = np.array([[r, d, lam, m.real, m.imag, c2b, float(ev)]
                                  for (r, d, lam, m, c2b, ev) in PLAIN])
    return out


def _config5_grains():
    """Seeded large, elongated grains: x uniform in [20, 30], axis ratio
    log-uniform in [0.33, 3], Re m in [1.3, 2], Im m log-uniform in
    [1e-3, 1], lambda = 1 um (equal-volume radii)."""
    rng = np.random.default_rng(505)
    n = 12
    x = rng.uniform(20.0, 30.0, n)
    d = np.exp(rng.uniform(np.log(0.33), np.log(3.0), n))
    m = rng.uniform(1.3, 2.0, n) + 1j * np.exp(rng.uniform(np.log(1e-3), 0.0, n))
    lam = 1e-6
    return x * lam / (2 * np.pi), lam, m, d


def _config5_one(i):
    """One grain through the reference module's TMatrix (calculator
    schedule, maximum_order 200, random orientation): its nmax and Z at
    181 scattering angles for incidence along the axis. Runs in a child
    process: the reference aborts the process when a grain does not
    converge."""
    r, lam, m, d = _config5_grains()
    C = O.ref_module()
    T = C.TMatrix(r[i], d[i], lam, m[i], cos2beta=1.0 / 3.0)
    tout = np.radians(np.arange(181.0))
    return T.get_nmax(), T.get_scattering_matrix(0.0, 0.0, tout, 0.0)


def _bench5_grains():
    """The 256 grains of bench.py's large-grain workload (seed 55): x
    uniform in [10, 30], axis ratio log-uniform in [0.33, 3]."""
    rng = np.random.default_rng(55)
    n = 256
    x = rng.uniform(10.0, 30.0, n)
    d = np.exp(rng.uniform(np.log(0.33), np.log(3.0), n))
    m = rng.uniform(1.3, 2.0, n) + 1j * np.exp(rng.uniform(np.log(1e-3), 0.0, n))
    lam = 1e-6
    return x * lam / (2 * np.pi), lam, m, d


def _bench5_one(i):
    """nmax of one bench grain from the reference module's TMatrix
    (calculator schedule, maximum_order 200, no orientation average)."""
    r, lam, m, d = _bench5_grains()
    T = O.ref_module().TMatrix(r[i], d[i], lam, m[i], cos2beta=-1.0)
    return T.get_nmax()


def _child(fn_name, i, q):
    q.put(globals()[fn_name](i))


def _isolated(fn_name, n, nproc=8):
    """fn(i) for i < n, each in a process of its own (at most nproc at a
    time), because the reference aborts the process when a grain does not
    converge. Returns the results, None where the process aborted."""
    import multiprocessing as mp
    import queue
    import time
    ctx = mp.get_context("spawn")
    out = [None] * n
    running = {}
    nxt = 0
    while nxt < n or running:
        while nxt < n and len(running) < nproc:
            q = ctx.Queue()
            p = ctx.Process(target=_child, args=(fn_name, nxt, q))
            p.start()
            running[nxt] = (p, q)
            nxt += 1
        for i in list(running):
            p, q = running[i]
            try:
                out[i] = q.get_nowait()
            except queue.Empty:
                if p.is_alive():
                    continue
                try:
                    out[i] = q.get(timeout=1)
                except queue.Empty:
                    pass  # aborted: not converged
            p.join()
            del running[i]
        time.sleep(0.2)
    return out


def config5():
    """Calculator-schedule outcomes of the reference module: for the seeded
    large grains, converged or aborted ("Unable to converge!"), nmax, and
    the random-orientation Z at 181 angles of the converged ones; for the
    256 grains of bench.py's large-grain workload, converged or aborted and
    nmax."""
    r, lam, m, d = _config5_grains()
    n = len(r)
    res = _isolated("_config5_one", n)
    conv = np.array([v is not None for v in res], np.int32)
    nmax = np.array([v[0] if v is not None else 0 for v in res], np.int32)
    Z = np.stack([v[1] if v is not None else np.zeros((181, 4, 4)) for v in res])
    rb, lamb, mb, db = _bench5_grains()
    resb = _isolated("_bench5_one", len(rb))
    return {"r_ev": r, "wavelength": np.array([lam]), "m": m, "d": d,
            "converged": conv, "nmax": nmax, "z181": Z,
            "bench_r_ev": rb, "bench_m": mb, "bench_d": db,
            "bench_converged": np.array([v is not None for v in resb], np.int32),
            "bench_nmax": np.array([v if v is not None else 0 for v in resb],
                                   np.int32)}


def _bench5_oracle_one(i):
    r, lam, m, d = _bench5_grains()
    return O.calculator_orders(r[i], lam, m[i], d[i])


def config5_oracle():
    """The C restatement's calculator orders (nmax, ngauss, status) for the
    256 grains of bench.py's large-grain workload, beside the reference
    module's in config5.npz: where the two differ, the convergence decision
    is set by rounding (the restatement follows the task path's operation
    order, the reference's TMatrix the plain path's)."""
    import multiprocessing as mp
    rb = _bench5_grains()[0]
    with mp.get_context("spawn").Pool(8) as p:
        res = p.map(_bench5_oracle_one, range(len(rb)))
    return {"bench_oracle": np.array(res, np.int32)}


def draine():
    """Refractive indices of the reference's DraineDustProperties (tabulated
    Draine 2003 optical constants from its data directory) for the three
    grain types at sizes 0.01-2 um and wavelengths across and beyond the
    tables (0.03 um - 300 um), at dust temperatures 20 K and 50 K."""
    C = O.ref_module()
    sizes = np.array([1e-8, 1e-7, 5e-7, 2e-6])
    lams = np.logspace(np.log10(3e-8), np.log10(3e-4), 41)
    out = {"sizes": sizes, "wavelengths": lams, "temperatures": np.array([20.0, 50.0])}
    for T in (20.0, 50.0):
        D = C.DraineDustProperties(dust_temperature=T)
        m = np.zeros((3, len(sizes), len(lams)), complex)
        for t in range(3):
            for i, a in enumerate(sizes):
                for j, lam in enumerate(lams):
                    m[t, i, j] = D.get_refractive_index(t, a, lam)
        out["m_%d" % int(T)] = m
    return out


if __name__ == "__main__":
    # python make_golden.py [stages tmatrices tables plain draine config5]: the named
    # sets (default all)
    which = sys.argv[1:] or ["stages", "tmatrices", "tables", "plain", "draine",
                             "config5", "config5_oracle"]
    for name in which:
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **globals()[name]())
    print("golden fixtures written to", HERE)
