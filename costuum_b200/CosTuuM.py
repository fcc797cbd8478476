"""Drop-in replacement of the CosTuuM Python module, computed on a B200.

Same names, arguments, defaults and outputs as the reference module
(src/CTMModule.cpp:146-541 and the src/Py*.hpp types); the work behind
``get_table`` runs through libtmx.so (include/tmx.h): T-matrices, orientation
averaging, extinction/absorption/scattering and shape averaging on the GPU,
in FP64.

Usage is unchanged::

    from costuum_b200 import CosTuuM
    Q = CosTuuM.get_table(types, sizes, wavelengths, thetas,
                          CosTuuM.DraineHensleyShapeDistribution(20),
                          CosTuuM.SizeBasedAlignmentDistribution(
                              1e-7, CosTuuM.MISHCHENKO_ALIGNMENT),
                          CosTuuM.CustomDustProperties(refractive_index))

Arguments that steered the reference's host scheduler (number_of_threads,
maximum_memory_size, the QuickSched and memory logs) are accepted; the GPU
schedule does not need them.
"""
import ctypes
import math
import os

import numpy as np

from . import _lib
from .tmatrix import default_context

DAVIS_GREENSTEIN_ALIGNMENT = 0
MISHCHENKO_ALIGNMENT = 1
DISABLE_ALIGNMENT = 2
CUSTOM_ALIGNMENT = 3

CARBON_PARALLEL = 0
CARBON_PERPENDICULAR = 1
SILICON = 2


def get_equal_volume_radius(radius, axis_ratio):
    """Equal-volume radius of a spheroid with the given equal-area radius."""
    return _lib.load().tmx_rv_over_rs(float(axis_ratio)) * float(radius)


# ------------------------------------------------------------------ shapes --

class _ShapeDistribution:
    def __init__(self, shapes, weights, limits):
        self._shapes = np.ascontiguousarray(shapes, np.float64)
        self._weights = np.ascontiguousarray(weights, np.float64)
        self._limits = (float(limits[0]), float(limits[1]))

    def get_limits(self):
        """(minimum, maximum) axis ratio of the distribution."""
        return self._limits

    @property
    def shapes(self):
        return self._shapes

    @property
    def weights(self):
        return self._weights


class SingleShapeShapeDistribution(_ShapeDistribution):
    """All grains share one axis ratio d = a / b."""

    def __init__(self, axis_ratio):
        d = float(axis_ratio)
        super().__init__([d], [1.0], (d, d))


class DraineHensleyShapeDistribution(_ShapeDistribution):
    """Draine & Hensley (2017) CDE2 shape distribution on npoints
    Gauss-Legendre nodes, limited by a probability cutoff or, if fraction > 0,
    by the prolate/oblate fraction it keeps."""

    def __init__(self, npoints=20, cutoff=0.15, fraction=-1.0):
        n = int(npoints)
        s = np.zeros(n)
        w = np.zeros(n)
        lim = np.zeros(2)
        rc = _lib.load().tmx_shape_distribution(1, n, float(cutoff), float(fraction),
                                                _lib.ptr(s), _lib.ptr(w), _lib.ptr(lim))
        if rc != 0:
            raise ValueError("invalid DraineHensleyShapeDistribution arguments")
        super().__init__(s, w, lim)


# ------------------------------------------------------------- orientation --

class _OrientationDistribution:
    """Expansion coefficients p_0..p_order of an orientation distribution."""

    compute_alignment = True

    def __init__(self, coefficients):
        self._coefficients = np.ascontiguousarray(coefficients, np.float64)

    @property
    def coefficients(self):
        return self._coefficients

    def get_maximum_order(self):
        return len(self._coefficients) - 1

    def evaluate(self, theta):
        """p(theta) = sum_n (2n + 1)/2 p_n d^n_00(theta), n < maximum order
        (PyOrientationDistribution::evaluate)."""
        th = np.atleast_1d(np.asarray(theta, np.float64))
        order = self.get_maximum_order()
        out = np.zeros_like(th)
        for i, t in enumerate(th):
            c = np.cos(t)
            d = np.zeros(max(order, 1))
            d[0] = 1.0
            if order > 1:
                d1, d2 = 1.0, c
                for n in range(order - 1):
                    d[n + 1] = d2
                    np1 = n + 1.0
                    d1, d2 = d2, ((2.0 * np1 + 1.0) * c * d2 - np1 * d1) / (n + 2.0)
            out[i] = sum(0.5 * (2.0 * n + 1.0) * self._coefficients[n] * d[n]
                         for n in range(order))
        return np.squeeze(out)


def _coefficients(kind, param, order, fn=None):
    out = np.zeros(int(order) + 1)
    lib = _lib.load()
    cb = _lib.ORIENT_FN(fn) if fn is not None else None
    rc = lib.tmx_orientation_coefficients(int(kind), float(param), int(order),
                                          ctypes.cast(cb, ctypes.c_void_p) if cb else None,
                                          None, _lib.ptr(out))
    if rc != 0:
        raise ValueError("invalid orientation distribution arguments")
    return out


class RandomOrientationDistribution(_OrientationDistribution):
    """Random orientation, p(beta) = 1/2 (coefficients by quadrature)."""

    def __init__(self, order=100):
        super().__init__(_coefficients(0, 0.0, order))


# the reference's C++ name for the random distribution
OrientationDistribution = RandomOrientationDistribution


class MishchenkoOrientationDistribution(_OrientationDistribution):
    """p(beta) = 1/2 + 5/4 p2 (3 cos^2 beta - 1), p2 = 3/2 cos2beta - 1/2."""

    def __init__(self, cos2beta, order=100):
        super().__init__(_coefficients(1, cos2beta, order))


class DavisGreensteinOrientationDistribution(_OrientationDistribution):
    """Perfect Davis-Greenstein alignment for the given axis ratio."""

    def __init__(self, axis_ratio, order=100):
        super().__init__(_coefficients(2, axis_ratio, order))


class CustomOrientationDistribution(_OrientationDistribution):
    """p(beta) given by a Python function function(beta[, additional_arguments])."""

    def __init__(self, function, order=100, additional_arguments=None):
        if additional_arguments is None:
            f = lambda b, _a: float(function(b))  # noqa: E731
        else:
            f = lambda b, _a: float(function(b, additional_arguments))  # noqa: E731
        super().__init__(_coefficients(3, 0.0, order, f))


class _DisabledAlignment(_OrientationDistribution):
    compute_alignment = False

    def __init__(self):
        super().__init__(np.zeros(1))


class SizeBasedAlignmentDistribution:
    """Grains larger than minimum_size align (oblate and prolate distributions
    by aligned_orientation_distribution_type); smaller grains orient randomly
    (SizeBasedAlignmentDistribution.hpp)."""

    def __init__(self, minimum_size, aligned_orientation_distribution_type,
                 maximum_order=100, oblate_orientation_distribution=None,
                 prolate_orientation_distribution=None):
        self.minimum_size = float(minimum_size)
        n = 2 * int(maximum_order)
        self.non_aligned = RandomOrientationDistribution(n)
        t = int(aligned_orientation_distribution_type)
        if t == DAVIS_GREENSTEIN_ALIGNMENT:
            self.oblate = DavisGreensteinOrientationDistribution(2.0, n)
            self.prolate = DavisGreensteinOrientationDistribution(0.5, n)
        elif t == MISHCHENKO_ALIGNMENT:
            self.oblate = MishchenkoOrientationDistribution(0.6, n)
            self.prolate = MishchenkoOrientationDistribution(0.2, n)
        elif t == DISABLE_ALIGNMENT:
            self.oblate = _DisabledAlignment()
            self.prolate = _DisabledAlignment()
        elif t == CUSTOM_ALIGNMENT:
            if oblate_orientation_distribution is None or \
                    prolate_orientation_distribution is None:
                raise ValueError("CUSTOM_ALIGNMENT needs oblate and prolate "
                                 "orientation distributions")
            # copies of the coefficients; averaging always on
            self.oblate = _OrientationDistribution(
                oblate_orientation_distribution.coefficients.copy())
            self.prolate = _OrientationDistribution(
                prolate_orientation_distribution.coefficients.copy())
        else:
            raise ValueError("Unknown orientation distribution!")

    def get_distribution(self, equal_volume_radius, axis_ratio):
        if equal_volume_radius > self.minimum_size:
            return self.oblate if axis_ratio > 1.0 else self.prolate
        return self.non_aligned


# -------------------------------------------------------------------- dust --

class CustomDustProperties:
    """Refractive index from function(wavelength, size, type[, arguments])."""

    def __init__(self, function, additional_arguments=None):
        self.function = function
        self.additional_arguments = additional_arguments

    def get_refractive_index(self, type, size, wavelength):
        if self.additional_arguments is None:
            v = self.function(wavelength, size, type)
        else:
            v = self.function(wavelength, size, type, self.additional_arguments)
        v = np.asarray(v)
        if v.size != 1 or not np.iscomplexobj(v):
            raise TypeError("Function does not return a complex number!")
        return complex(v.reshape(()))


def _read_index_table(path):
    """Rows of a Draine optical-constant file: every line that does not start
    with '#', five columns (wavelength in micron, eps_1 - 1, eps_2,
    Re(n) - 1, Im(n)); Table::from_ascii_file (Table.hpp:126-142)."""
    rows = []
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            parts = line.split()
            if len(parts) < 5:
                continue
            rows.append([float(v) for v in parts[:5]])
    return rows


def _interpolated_row(rows, x):
    """Linear interpolation of every column at column-0 value x: bisection
    for the bracketing rows (increasing or decreasing column 0), then
    (1 - f) row_low + f row_high with f = (x - x_low) / (x_high - x_low);
    outside the table the end pair is extrapolated
    (LinearInterpolatedTable::get_row, Table.hpp:201-260)."""
    lo, hi = 0, len(rows) - 1
    xlo, xhi = rows[lo][0], rows[hi][0]
    if xlo == xhi:
        raise ValueError("Table endpoints are the same!")
    increasing = xlo < xhi
    while lo + 1 != hi:
        mid = (lo + hi) >> 1
        xm = rows[mid][0]
        if (xm <= x) if increasing else (xm >= x):
            xlo, lo = xm, mid
        else:
            xhi, hi = xm, mid
    f = (x - xlo) / (xhi - xlo)
    return [(1.0 - f) * a + f * b for a, b in zip(rows[lo], rows[hi])]


def _carbon_free_electron_eps(T, wavelength, grain_size, parallel):
    """Free-electron term of the graphite dielectric function (Draine & Lee
    1984, eq. 2.2 with table 1 and the 1987 erratum; size dependence of the
    damping time by eqs. 2.5-2.6), as DraineDustProperties::get_C_epsilon_free
    (DraineDustProperties.hpp:73-107) evaluates it."""
    if parallel:
        omega_p, tau_bulk, TF, vF = 1.53e14, 1.4e-14, 255.0, 3.7e4
    else:
        T2 = T * T
        omega_p = 4.33e14 * math.sqrt(1.0 - 6.24e-3 * T + 3.66e-5 * T2)
        tau_bulk = 4.2e-11 / (1.0 + 0.322 * T + 0.0013 * T2)
        TF, vF = 255.0, 4.5e5
    veff = vF * math.sqrt(1.0 + T / TF)
    tau = 1.0 / (1.0 / tau_bulk + veff / grain_size)
    omega = 2.0 * math.pi * 299792458.0 / wavelength
    wt = omega * tau
    wpt = omega_p * tau
    return complex(-wpt * wpt, 0.0) / complex(wt * wt, wt)


def _eps_to_refractive_index(eps):
    """n = sqrt((|eps| + eps_r) / 2) + i sqrt((|eps| - eps_r) / 2)
    (DraineDustProperties::eps_to_mr, DraineDustProperties.hpp:133-139)."""
    er, ei = eps.real, eps.imag
    a = math.sqrt(er * er + ei * ei)
    return complex(math.sqrt(0.5 * (a + er)), math.sqrt(0.5 * (a - er)))


class DraineDustProperties:
    """Refractive indices of Draine (2003) astrosilicate and graphite (E
    parallel and perpendicular to the c axis) from the tabulated optical
    constants that the reference ships in its data directory
    (DraineDustProperties.hpp:36-242): linear interpolation in wavelength,
    and for graphite the free-electron term of the dielectric function
    re-evaluated for the grain's size and the dust temperature (the tables
    include it for 20 K and 0.1 micron).

    The tables are not part of this package. data_directory (or the
    environment variable COSTUUM_DRAINE_DATA) names the directory that holds
    the reference's files callindex.out_silD03, callindex.out_CpaD03_0.10 and
    callindex.out_CpeD03_0.10."""

    FILES = {SILICON: "callindex.out_silD03",
             CARBON_PARALLEL: "callindex.out_CpaD03_0.10",
             CARBON_PERPENDICULAR: "callindex.out_CpeD03_0.10"}

    def __init__(self, dust_temperature=20.0, data_directory=None):
        self.dust_temperature = float(dust_temperature)
        d = data_directory or os.environ.get("COSTUUM_DRAINE_DATA")
        if not d:
            raise FileNotFoundError(
                "DraineDustProperties reads the tabulated Draine (2003) optical "
                "constants (%s); pass data_directory= or set COSTUUM_DRAINE_DATA "
                "to the directory that holds them" % ", ".join(sorted(self.FILES.values())))
        self._tables = {}
        for kind, name in self.FILES.items():
            path = os.path.join(d, name)
            if not os.path.isfile(path):
                raise FileNotFoundError("Unable to open file: \"%s\"!" % path)
            rows = _read_index_table(path)
            for r in rows:
                r[0] *= 1e-6   # micron -> m
                r[1] += 1.0    # eps_1
                r[3] += 1.0    # Re(n)
            if kind != SILICON:
                # remove the free-electron term of the tabulated 20 K, 0.1 um
                parallel = kind == CARBON_PARALLEL
                for r in rows:
                    c = _carbon_free_electron_eps(20.0, r[0], 1e-7, parallel)
                    r[1] -= c.real
                    r[2] -= c.imag
            self._tables[kind] = rows

    def get_refractive_index(self, type, size, wavelength):
        type = int(type)
        if type not in self._tables:
            raise ValueError("Unknown dust grain type: %d!" % type)
        row = _interpolated_row(self._tables[type], float(wavelength))
        if type == SILICON:
            return complex(row[3], row[4])
        eps = complex(row[1], row[2]) + _carbon_free_electron_eps(
            self.dust_temperature, float(wavelength), float(size),
            type == CARBON_PARALLEL)
        return _eps_to_refractive_index(eps)


# --------------------------------------------------------------- get_table --

def get_table(types, sizes, wavelengths, thetas, shape_distribution,
              alignment_distribution, dust_properties, minimum_order=10,
              maximum_order=100, gauss_legendre_factor=2, tolerance=1e-4,
              number_of_quadrature_angles=20, maximum_memory_size=10000000000,
              number_of_threads=4, quicksched_graph_log=None,
              quicksched_task_log=None, quicksched_task_type_log=None,
              memory_log=None, do_absorption=True, do_extinction=False,
              do_scattering=False, account_for_scattering=False, verbose=False,
              return_status=False, context=None):
    """Absorption/extinction coefficients and/or scattering matrices averaged
    over shape and orientation (CTMModule.cpp:146-478).

    Returns a squeezed float64 array [type, size, wavelength, theta, k] with
    k = (Qabs, Qabspol) if do_absorption followed by (Qext, Qextpol,
    Qextcpol) if do_extinction, and/or a squeezed array [type, size,
    wavelength, theta, 2 theta, 4, 4] of scattering matrices; a tuple if
    both. Sizes and wavelengths are sorted (as the reference does).
    With return_status=True the per-grain status bits
    [type, size, wavelength, shape] are appended to the result."""
    ctx = context if context is not None else default_context()
    types = np.atleast_1d(np.asarray(types)).astype(np.int64)
    sizes = np.sort(np.atleast_1d(np.asarray(sizes, np.float64)))
    lams = np.sort(np.atleast_1d(np.asarray(wavelengths, np.float64)))
    thetas = np.ascontiguousarray(np.atleast_1d(np.asarray(thetas, np.float64)))
    nt, ns, nl, nth = len(types), len(sizes), len(lams), len(thetas)
    shapes = shape_distribution.shapes
    wts = shape_distribution.weights
    nsh = len(shapes)
    # refractive index per (type, size, wavelength), as TaskManager asks for it
    mr = np.zeros((nt, ns, nl))
    mi = np.zeros((nt, ns, nl))
    for it, t in enumerate(types):
        for isz, s in enumerate(sizes):
            for il, lam in enumerate(lams):
                v = dust_properties.get_refractive_index(int(t), float(s), float(lam))
                mr[it, isz, il] = v.real
                mi[it, isz, il] = v.imag
    # orientation coefficient sets per (size, shape)
    sets, index = [], {}
    orient = np.zeros((ns, nsh), np.int32)
    for isz, s in enumerate(sizes):
        for ish, d in enumerate(shapes):
            od = alignment_distribution.get_distribution(float(s), float(d))
            if not od.compute_alignment:
                orient[isz, ish] = -1
                continue
            key = id(od)
            if key not in index:
                index[key] = len(sets)
                sets.append(od.coefficients)
            orient[isz, ish] = index[key]
    ncoef = max([len(c) for c in sets] + [2 * int(maximum_order) + 1])
    coeffs = np.zeros((max(1, len(sets)), ncoef))
    for i, c in enumerate(sets):
        coeffs[i, :len(c)] = c
    flags = ((1 if do_absorption else 0) | (2 if do_extinction else 0)
             | (4 if do_scattering else 0) | (8 if account_for_scattering else 0))
    nq = (2 if do_absorption else 0) + (3 if do_extinction else 0)
    out_q = np.zeros((nt, ns, nl, nth, max(nq, 1)))
    out_z = np.zeros((nt, ns, nl, nth, 2 * nth, 4, 4)) if do_scattering else np.zeros(1)
    status = np.zeros((nt, ns, nl, nsh), np.int32)
    sched = _lib.TmxSchedule(int(minimum_order), int(maximum_order),
                             int(gauss_legendre_factor), 0, float(tolerance))
    lib = _lib.load()
    mr = np.ascontiguousarray(mr)
    mi = np.ascontiguousarray(mi)
    orient = np.ascontiguousarray(orient)
    with ctx._lock:
        rc = lib.tmx_get_table(ctx._h, nt, ns, _lib.ptr(sizes), nl, _lib.ptr(lams),
                               nth, _lib.ptr(thetas), nsh, _lib.ptr(shapes),
                               _lib.ptr(wts), _lib.ptr(mr), _lib.ptr(mi),
                               _lib.iptr(orient), len(sets), _lib.ptr(coeffs),
                               ncoef, flags, int(number_of_quadrature_angles),
                               ctypes.byref(sched),
                               _lib.ptr(out_q) if nq else None,
                               _lib.ptr(out_z) if do_scattering else None,
                               _lib.iptr(status))
        ctx._batch_id = ctx.batch_id + 1  # the grid's batches replaced the last one
        _lib.check(ctx._h, rc, "tmx_get_table")
    res = []
    if nq:
        res.append(np.squeeze(out_q[..., :nq]))
    if do_scattering:
        res.append(np.squeeze(out_z))
    if return_status:
        res.append(status)
    if len(res) == 1:
        return res[0]
    return tuple(res)


# ----------------------------------------------------------- plain path --

class TMatrix:
    """One particle's T-matrix on the plain path (CosTuuM.TMatrix,
    PyTMatrix.hpp:118-227): converged with the calculator schedule
    (TMatrixCalculator::calculate_TMatrix), then, for cos2beta >= 0,
    averaged over the orientation distribution with expansion order
    2 nmax: Davis-Greenstein for cos2beta 0 or 1, random orientation for
    1/3, Mishchenko otherwise. Each object keeps its T-matrix on the GPU in
    a context of its own. Angles are in radians, lengths in metres.
    """

    def __init__(self, particle_radius, axis_ratio, wavelength, refractive_index,
                 cos2beta=1.0 / 3.0, tolerance=1e-4, maximum_order=200,
                 gauss_legendre_factor=2, maximum_ngauss=500,
                 is_equal_volume_radius=True):
        from .tmatrix import Context
        r = float(particle_radius)
        if not is_equal_volume_radius:
            r = get_equal_volume_radius(r, axis_ratio)
        self._ctx = Context(0)
        res = self._ctx.tmatrix_batch_calculator(
            [r], float(wavelength), complex(refractive_index), float(axis_ratio),
            maximum_order=maximum_order, tolerance=tolerance,
            gauss_legendre_factor=gauss_legendre_factor,
            maximum_ngauss=maximum_ngauss)
        self._status = int(res.status[0])
        if self._status & ~1:
            raise RuntimeError("T-matrix calculation failed (status %d)" % self._status)
        self._nmax = int(res.nmax[0])
        self._ngauss = int(res.ngauss[0])
        self._q = res.q[0].copy()
        if cos2beta >= 0.0:
            order = 2 * self._nmax
            if cos2beta == 0.0 or cos2beta == 1.0:
                od = DavisGreensteinOrientationDistribution(axis_ratio, order)
            elif cos2beta == 1.0 / 3.0:
                od = RandomOrientationDistribution(order)
            else:
                od = MishchenkoOrientationDistribution(cos2beta, order)
            self._ctx.orientation_average(od.coefficients, [0])

    @property
    def converged(self):
        """False where the reference would have aborted ("Unable to
        converge!"): the order or quadrature limit was reached."""
        return self._status == 0

    def get_nmax(self):
        return self._nmax

    def get_ngauss(self):
        return self._ngauss

    def get_extinction_matrix(self, theta, phi, alpha=0.0, beta=0.0):
        """K[theta, phi, 4, 4], squeezed."""
        th = np.atleast_1d(np.asarray(theta, np.float64)).ravel()
        ph = np.atleast_1d(np.asarray(phi, np.float64)).ravel()
        T, P = np.meshgrid(th, ph, indexing="ij")
        K = self._ctx.extinction_matrix(0, T, P, alpha, beta)
        return np.squeeze(K)

    def get_scattering_matrix(self, theta_in, phi_in, theta_out, phi_out,
                              alpha=0.0, beta=0.0):
        """Z[theta_in, phi_in, theta_out, phi_out, 4, 4], squeezed."""
        a = [np.atleast_1d(np.asarray(x, np.float64)).ravel()
             for x in (theta_in, phi_in, theta_out, phi_out)]
        grids = np.meshgrid(*a, indexing="ij")
        Z = self._ctx.scattering_matrix(0, grids[0], grids[1], grids[2], grids[3],
                                        alpha, beta)
        return np.squeeze(Z)

    def get_absorption_cross_section(self, theta, ngauss=100):
        """Cabs for each zenith angle (1D array)."""
        th = np.atleast_1d(np.asarray(theta, np.float64)).ravel()
        return self._ctx.absorption_cross_sections(0, th, ngauss)[:, 0].copy()

    def get_absorption_cross_sections(self, theta, ngauss=100):
        """(Cabs, Cabspol) for each zenith angle, squeezed."""
        th = np.atleast_1d(np.asarray(theta, np.float64)).ravel()
        return np.squeeze(self._ctx.absorption_cross_sections(0, th, ngauss))

    def get_average_absorption_cross_section(self):
        return self._ctx.average_absorption_cross_section(0, 20)
