"""ctypes bindings for the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Two libraries sit behind this module:

* ``liboracle.so`` (oracle/tmx_oracle.c): the plain-C restatement of the
  CosTuuM reference algorithms. It is the checker the CUDA path is compared
  with.
* ``_ref/libref_driver.so`` and ``_ref/CosTuuM*.so`` (oracle/build_ref.sh):
  the unmodified reference, compiled from its own sources. It pins the
  restatement and serves as the timed CPU baseline. It exists wherever the
  build ran (it travels with the repository's built files); ``have_ref()``
  says whether it is present.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
import ctypes
import glob
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _p(a):
    return a.ctypes.data_as(_D)


def _cplx(a):
    """Interleaved (re, im) float64 view of a complex128 array."""
    return np.ascontiguousarray(a, dtype=np.complex128)


_lib = None


def lib():
    """The C restatement (builds nothing; call ``make -C oracle`` first)."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so missing: run make -C oracle")
        L = ctypes.CDLL(path)
        L.or_gauss_legendre.argtypes = [ctypes.c_int, _D, _D]
        L.or_bessel_j_real.argtypes = [ctypes.c_int, ctypes.c_double, _D, _D]
        L.or_bessel_y_real.argtypes = [ctypes.c_int, ctypes.c_double, _D, _D]
        L.or_bessel_j_complex.argtypes = [ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, _D, _D]
        L.or_bessel_j_real_start.argtypes = [ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, _D, _D]
        L.or_bessel_j_complex_start.argtypes = [ctypes.c_int, ctypes.c_int,
                                                ctypes.c_double, ctypes.c_double,
                                                _D, _D]
        L.or_wigner_d.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                  _D, _D]
        L.or_wigner_d_sinx.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int] * 2 + [_D, _D]
        L.or_rv_over_rs.argtypes = [ctypes.c_double]
        L.or_rv_over_rs.restype = ctypes.c_double
        L.or_clebsch_gordan_row.argtypes = [ctypes.c_int] * 3 + [_D]
        L.or_clebsch_gordan_row.restype = ctypes.c_int
        L.or_plu_inverse.argtypes = [ctypes.c_int, _D]
        L.or_orientation_coefficients.argtypes = [ctypes.c_int, ctypes.c_double,
                                                  ctypes.c_int, _D]
        L.or_tmatrix_size.argtypes = [ctypes.c_int]
        L.or_tmatrix_size.restype = ctypes.c_long
        L.or_tmatrix_block_offset.argtypes = [ctypes.c_int, ctypes.c_int]
        L.or_tmatrix_block_offset.restype = ctypes.c_long
        L.or_tmatrix_m0.argtypes = [ctypes.c_double] * 5 + [ctypes.c_int] * 2 + [_D, _D, _D]
        L.or_tmatrix_mblock.argtypes = [ctypes.c_double] * 5 + [ctypes.c_int] * 3 + [_D]
        L.or_tmatrix_converge.argtypes = ([ctypes.c_double] * 5 + [ctypes.c_int] * 3
                                          + [ctypes.c_double, _D, _I, _I, _D])
        L.or_tmatrix_converge.restype = ctypes.c_int
        L.or_tmatrix_q.argtypes = [ctypes.c_int, _D, _D, _D]
        L.or_orientation_average.argtypes = [ctypes.c_int, _D, _D, _D]
        L.or_extinction.argtypes = [ctypes.c_int, _D, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, _D, _D]
        L.or_absorption.argtypes = [ctypes.c_int, _D, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, _D,
                                    ctypes.c_int, ctypes.c_int, _D]
        L.or_scattering_matrix.argtypes = [ctypes.c_int, _D, ctypes.c_double,
                                           ctypes.c_int, _D]
        L.or_calculator_orders.argtypes = ([ctypes.c_double] * 5 + [ctypes.c_int,
                                           ctypes.c_double, ctypes.c_int,
                                           ctypes.c_int, _I, _I])
        L.or_calculator_orders.restype = ctypes.c_int
        L.or_amplitude_lab.argtypes = [ctypes.c_int, _D] + [ctypes.c_double] * 7 + [_D]
        L.or_z_from_s.argtypes = [_D, _D]
        L.or_k_from_s.argtypes = [ctypes.c_double, _D, _D]
        _lib = L
    return _lib


# ------------------------------------------------------------ restatement ---

def gauss_legendre(order):
    x = np.zeros(order)
    w = np.zeros(order)
    lib().or_gauss_legendre(order, _p(x), _p(w))
    return x, w


def bessel_j_real(nmax, z):
    j = np.zeros(nmax)
    dj = np.zeros(nmax)
    lib().or_bessel_j_real(nmax, z, _p(j), _p(dj))
    return j, dj


def bessel_y_real(nmax, z):
    y = np.zeros(nmax)
    dy = np.zeros(nmax)
    lib().or_bessel_y_real(nmax, z, _p(y), _p(dy))
    return y, dy


def bessel_j_complex(nmax, z):
    j = np.zeros(nmax, np.complex128)
    dj = np.zeros(nmax, np.complex128)
    lib().or_bessel_j_complex(nmax, z.real, z.imag, _p(j), _p(dj))
    return j, dj


def bessel_j_real_start(nmax, start, z):
    j = np.zeros(nmax)
    dj = np.zeros(nmax)
    lib().or_bessel_j_real_start(nmax, start, z, _p(j), _p(dj))
    return j, dj


def bessel_j_complex_start(nmax, start, z):
    j = np.zeros(nmax, np.complex128)
    dj = np.zeros(nmax, np.complex128)
    lib().or_bessel_j_complex_start(nmax, start, z.real, z.imag, _p(j), _p(dj))
    return j, dj


def wigner_d(cosx, nmax, m):
    d = np.zeros(nmax)
    dd = np.zeros(nmax)
    lib().or_wigner_d(cosx, nmax, m, _p(d), _p(dd))
    return d, dd


def wigner_d_sinx(cosx, sinx, sinx_inv, nmax, m):
    d = np.zeros(nmax)
    dd = np.zeros(nmax)
    lib().or_wigner_d_sinx(cosx, sinx, sinx_inv, nmax, m, _p(d), _p(dd))
    return d, dd


def rv_over_rs(d):
    return lib().or_rv_over_rs(d)


def clebsch_gordan_row(n1, n2, N):
    out = np.zeros(2 * min(n1, n2) + 1)
    lib().or_clebsch_gordan_row(n1, n2, N, _p(out))
    return out


def plu_inverse(a):
    a = _cplx(a).copy()
    lib().or_plu_inverse(a.shape[0], _p(a))
    return a


def orientation_coefficients(kind, param, order):
    out = np.zeros(order + 1)
    lib().or_orientation_coefficients(kind, param, order, _p(out))
    return out


def tmatrix_size(nmax):
    """Number of complex elements of a full T-matrix (all m blocks)."""
    return lib().or_tmatrix_size(nmax) // 2


def block_offset(nmax, m):
    """Complex-element offset of block m."""
    return lib().or_tmatrix_block_offset(nmax, m) // 2


def block(T, nmax, m):
    """Block m of a flat T-matrix as a (2nb, 2nb) complex matrix."""
    nb = nmax if m == 0 else nmax + 1 - m
    off = block_offset(nmax, m)
    return T[off:off + 4 * nb * nb].reshape(2 * nb, 2 * nb)


def tmatrix_m0(r_ev, wavelength, m, d, nmax, ngauss):
    T0 = np.zeros((2 * nmax, 2 * nmax), np.complex128)
    qs = np.zeros(1)
    qe = np.zeros(1)
    lib().or_tmatrix_m0(r_ev, wavelength, m.real, m.imag, d, nmax, ngauss,
                        _p(T0), _p(qs), _p(qe))
    return T0, qs[0], qe[0]


def tmatrix_mblock(r_ev, wavelength, m, d, nmax, ngauss, mm):
    nb = nmax if mm == 0 else nmax + 1 - mm
    T = np.zeros((2 * nb, 2 * nb), np.complex128)
    lib().or_tmatrix_mblock(r_ev, wavelength, m.real, m.imag, d, nmax, ngauss,
                            mm, _p(T))
    return T


def tmatrix_converge(r_ev, wavelength, m, d, min_order=10, max_order=100,
                     glfac=2, tolerance=1e-4):
    """Task-based (TaskManager) schedule for one grain.

    Returns dict(nmax, ngauss, converged, T (flat complex), info)."""
    T = np.zeros(tmatrix_size(max_order), np.complex128)
    ng = ctypes.c_int(0)
    conv = ctypes.c_int(0)
    info = np.zeros(6)
    nmax = lib().or_tmatrix_converge(r_ev, wavelength, m.real, m.imag, d,
                                     min_order, max_order, glfac, tolerance,
                                     _p(T), ctypes.byref(ng), ctypes.byref(conv),
                                     _p(info))
    return dict(nmax=nmax, ngauss=ng.value, converged=bool(conv.value),
                T=T[:tmatrix_size(nmax)].copy(), info=info)


def tmatrix_q(T, nmax):
    qs = np.zeros(1)
    qe = np.zeros(1)
    lib().or_tmatrix_q(nmax, _p(_cplx(T)), _p(qs), _p(qe))
    return qs[0], qe[0]


def orientation_average(T, nmax, coeffs):
    T = _cplx(T)
    Ta = np.zeros_like(T)
    c = None if coeffs is None else np.ascontiguousarray(coeffs, np.float64)
    lib().or_orientation_average(nmax, _p(T), None if c is None else _p(c),
                                 _p(Ta))
    return Ta


def extinction(T, nmax, wavelength, r_ev, theta):
    theta = np.ascontiguousarray(theta, np.float64)
    out = np.zeros((len(theta), 3))
    lib().or_extinction(nmax, _p(_cplx(T)), wavelength, r_ev, len(theta),
                        _p(theta), _p(out))
    return out


def absorption(T, nmax, wavelength, r_ev, theta, ngauss=20,
               account_for_scattering=False):
    theta = np.ascontiguousarray(theta, np.float64)
    out = np.zeros((len(theta), 2))
    lib().or_absorption(nmax, _p(_cplx(T)), wavelength, r_ev, len(theta),
                        _p(theta), ngauss, int(account_for_scattering), _p(out))
    return out


def calculator_orders(r_ev, wavelength, m, d, maximum_order=200, tolerance=1e-4,
                      ndgs=2, maximum_ngauss=500):
    """Plain-path (TMatrixCalculator) orders: (nmax, ngauss, status)."""
    nm = ctypes.c_int(0)
    ng = ctypes.c_int(0)
    st = lib().or_calculator_orders(r_ev, wavelength, m.real, m.imag, d,
                                    maximum_order, tolerance, ndgs, maximum_ngauss,
                                    ctypes.byref(nm), ctypes.byref(ng))
    return nm.value, ng.value, st


def full_tmatrix(r_ev, wavelength, m, d, nmax, ngauss):
    """Every block at (nmax, ngauss), flat complex in the block layout."""
    T = np.zeros(tmatrix_size(nmax), np.complex128)
    T0, _, _ = tmatrix_m0(r_ev, wavelength, m, d, nmax, ngauss)
    T[:4 * nmax * nmax] = T0.ravel()
    for mm in range(1, nmax + 1):
        o = block_offset(nmax, mm)
        blk = tmatrix_mblock(r_ev, wavelength, m, d, nmax, ngauss, mm)
        T[o:o + blk.size] = blk.ravel()
    return T


def amplitude_lab(T, nmax, wavelength, alpha, beta, theta_in, phi_in, theta_out,
                  phi_out):
    S = np.zeros((2, 2), np.complex128)
    lib().or_amplitude_lab(nmax, _p(_cplx(T)), wavelength, alpha, beta, theta_in,
                           phi_in, theta_out, phi_out, _p(S))
    return S


def z_from_s(S):
    Z = np.zeros((4, 4))
    lib().or_z_from_s(_p(np.ascontiguousarray(S, np.complex128)), _p(Z))
    return Z


def k_from_s(wavelength, S):
    K = np.zeros((4, 4))
    lib().or_k_from_s(wavelength, _p(np.ascontiguousarray(S, np.complex128)), _p(K))
    return K


def scattering_matrix(T, nmax, wavelength, ntheta):
    out = np.zeros((ntheta, 2 * ntheta, 4, 4))
    lib().or_scattering_matrix(nmax, _p(_cplx(T)), wavelength, ntheta, _p(out))
    return out


# ------------------------------------------------------ reference (built) ---

_ref = None


def have_ref():
    return os.path.exists(os.path.join(HERE, "_ref", "libref_driver.so"))


def ref():
    """The unmodified reference's task objects behind a C ABI."""
    global _ref
    if _ref is None:
        L = ctypes.CDLL(os.path.join(HERE, "_ref", "libref_driver.so"))
        L.ref_gauss_legendre.argtypes = [ctypes.c_int, _D, _D]
        L.ref_bessel_j_real.argtypes = [ctypes.c_int, ctypes.c_double, _D, _D]
        L.ref_bessel_y_real.argtypes = [ctypes.c_int, ctypes.c_double, _D, _D]
        L.ref_bessel_j_complex.argtypes = [ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, _D, _D]
        L.ref_wigner_d.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                   _D, _D]
        L.ref_wigner_d_sinx.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int] * 2 + [_D, _D]
        L.ref_rv_over_rs.argtypes = [ctypes.c_double]
        L.ref_rv_over_rs.restype = ctypes.c_double
        L.ref_clebsch_gordan_row.argtypes = [ctypes.c_int] * 3 + [_D]
        L.ref_clebsch_gordan_row.restype = ctypes.c_int
        L.ref_plu_inverse.argtypes = [ctypes.c_int, _D]
        L.ref_orientation_coefficients.argtypes = [ctypes.c_int, ctypes.c_double,
                                                   ctypes.c_int, _D]
        L.ref_custom_orientation_coefficients.argtypes = [ctypes.c_int, _D]
        L.ref_draine_hensley.argtypes = [ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, _D, _D, _D]
        L.ref_batch_create.restype = ctypes.c_void_p
        L.ref_batch_create.argtypes = ([ctypes.c_int] + [_D] * 5 + [ctypes.c_int] * 3
                                       + [ctypes.c_double, ctypes.c_int])
        L.ref_batch_run.argtypes = [ctypes.c_void_p]
        L.ref_batch_destroy.argtypes = [ctypes.c_void_p]
        L.ref_batch_nmax.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_batch_ngauss.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_batch_converged.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_batch_q.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
        L.ref_batch_tblock.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_int, _D]
        _ref = L
    return _ref


def draine_data_directory():
    """Directory of the reference's tabulated Draine optical constants, as
    recorded by build_ref.sh in the generated DraineDustPropertiesDataLocation
    header; None where the reference build or its data are absent."""
    h = os.path.join(HERE, "_ref", "gen", "DraineDustPropertiesDataLocation.hpp")
    if not os.path.isfile(h):
        return None
    with open(h) as f:
        for line in f:
            if line.startswith("#define DRAINEDUSTPROPERTIESDATALOCATION "):
                d = line.split('"')[1]
                return d if os.path.isdir(d) else None
    return None


def ref_module():
    """The reference's own CPython module (CosTuuM), built by build_ref.sh."""
    d = os.path.join(HERE, "_ref")
    if d not in sys.path:
        sys.path.insert(0, d)
    import CosTuuM  # noqa: E402
    return CosTuuM


def ref_batch(r_ev, wavelength, m, d, min_order=10, max_order=100, glfac=2,
              tolerance=1e-4, nthreads=1, want_t=True):
    """Run independent grains through the reference's task objects under
    QuickSched. Returns a list of dicts (nmax, ngauss, converged, q, T)."""
    R = ref()
    r_ev = np.ascontiguousarray(r_ev, np.float64)
    wavelength = np.ascontiguousarray(wavelength, np.float64)
    m = np.asarray(m, np.complex128)
    mr = np.ascontiguousarray(m.real)
    mi = np.ascontiguousarray(m.imag)
    d = np.ascontiguousarray(d, np.float64)
    n = len(r_ev)
    h = R.ref_batch_create(n, _p(r_ev), _p(wavelength), _p(mr), _p(mi), _p(d),
                           min_order, max_order, glfac, tolerance, nthreads)
    R.ref_batch_run(h)
    out = []
    for g in range(n):
        nmax = R.ref_batch_nmax(h, g)
        q = np.zeros(6)
        R.ref_batch_q(h, g, _p(q))
        rec = dict(nmax=nmax, ngauss=R.ref_batch_ngauss(h, g),
                   converged=bool(R.ref_batch_converged(h, g)), q=q)
        if want_t:
            T = np.zeros(tmatrix_size(nmax), np.complex128)
            for mm in range(nmax + 1):
                nb = nmax if mm == 0 else nmax + 1 - mm
                blk = np.zeros((2 * nb, 2 * nb), np.complex128)
                R.ref_batch_tblock(h, g, mm, _p(blk))
                off = block_offset(nmax, mm)
                T[off:off + 4 * nb * nb] = blk.ravel()
            rec["T"] = T
        out.append(rec)
    R.ref_batch_destroy(h)
    return out
