"""Batched T-matrices of independent spheroids on the GPU.

This is the Python face of the C ABI in include/tmx.h. A batch runs the
reference's task-based schedule (CosTuuM TaskManager: orders min_order ..
max_order - 1 with ngauss = gauss_legendre_factor * order until the m = 0
Qsca and Qext converge, then every m block) for every grain at once.
"""
import ctypes
import threading
import weakref

import numpy as np

from . import _lib

GRAIN_OK = 0
GRAIN_NOT_CONVERGED = 1
GRAIN_SINGULAR = 2
GRAIN_NAN = 4
GRAIN_BAD_INPUT = 8
GRAIN_TOO_LARGE = 16


def tmatrix_size(nmax):
    """Complex elements of a T-matrix holding every m block up to nmax."""
    return int(_lib.load().tmx_tmatrix_size(int(nmax)))


def block_offset(nmax, m):
    """Complex offset of block m inside a flat T-matrix."""
    if m == 0:
        return 0
    nb = np.arange(nmax + 1 - (m - 1), nmax + 1)
    return int(4 * nmax * nmax + 4 * int(np.sum(nb.astype(np.int64) ** 2)))


def block(T, nmax, m):
    """Block m of a flat T-matrix as a (2nb, 2nb) complex matrix."""
    nb = nmax if m == 0 else nmax + 1 - m
    off = block_offset(nmax, m)
    return T[off:off + 4 * nb * nb].reshape(2 * nb, 2 * nb)


class BatchResult:
    """Per-grain outcome of Context.tmatrix_batch."""

    def __init__(self, ctx, n, nmax, ngauss, status, q):
        self._ctx = ctx
        self.n = n
        self.nmax = nmax
        self.ngauss = ngauss
        self.status = status
        self.q = q  # [m0 Qsca, m0 Qext, full Qsca, full Qext, dQs, dQe]

    @property
    def qsca(self):
        return self.q[:, 2]

    @property
    def qext(self):
        return self.q[:, 3]

    def tmatrix(self, i):
        """Flat complex T-matrix of grain i (reference block layout)."""
        N = int(self.nmax[i])
        out = np.zeros(tmatrix_size(N), np.complex128)
        if N > 0:
            rc = _lib.load().tmx_batch_tmatrix(self._ctx._h, int(i), _lib.ptr(out))
            _lib.check(self._ctx._h, rc, "tmx_batch_tmatrix")
        return out


class _PinnedPool:
    """Page-locked host buffers for result arrays. A result views a pooled
    buffer; the buffer returns to the pool when the last view of it is
    released, so repeated calls reuse the same page-locked memory and their
    device-to-host copies run as direct DMA."""

    def __init__(self):
        self._free = []  # (capacity, address)
        self._closed = False

    def _release(self, cap, ptr):
        if self._closed:
            _lib.load().tmx_host_free(ptr)
        else:
            self._free.append((cap, ptr))

    def array(self, shape):
        count = int(np.prod(shape))
        nbytes = max(8, 8 * count)
        pick = None
        for i, (cap, ptr) in enumerate(self._free):
            if cap >= nbytes and (pick is None or cap < self._free[pick][0]):
                pick = i
        if pick is not None:
            cap, ptr = self._free.pop(pick)
        else:
            cap = max(nbytes, 1 << 16)
            ptr = _lib.load().tmx_host_alloc(cap)
            if not ptr:
                return np.empty(shape)  # pageable fallback
        buf = (ctypes.c_char * cap).from_address(ptr)
        weakref.finalize(buf, self._release, cap, ptr)
        return np.frombuffer(buf, dtype=np.float64, count=count).reshape(shape)

    def close(self):
        self._closed = True
        lib = _lib.load()
        for _, ptr in self._free:
            lib.tmx_host_free(ptr)
        self._free = []


class Context:
    """A CUDA device context: owns device buffers and cached tables."""

    def __init__(self, device=0):
        lib = _lib.load()
        h = ctypes.c_void_p()
        rc = lib.tmx_create(ctypes.byref(h), int(device))
        if rc != 0:
            raise _lib.TmxError("tmx_create failed (%d): no usable CUDA device "
                                "or CUDA error" % rc)
        self._h = h
        self.device = device
        self._lock = threading.Lock()
        self._pinned = _PinnedPool()

    def close(self):
        if getattr(self, "_pinned", None):
            self._pinned.close()
        if getattr(self, "_h", None):
            _lib.load().tmx_destroy(self._h)
            self._h = None
        if getattr(self, "_sink", None):
            _lib.load().tmx_host_free(self._sink[0])
            self._sink = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def kernel_launches(self):
        return int(_lib.load().tmx_kernel_launches(self._h))

    def probe_fp64(self, kind=0):
        """Measured FP64 TFLOP/s: kind 0 DFMA pipe, 1 DMMA tensor pipe."""
        v = np.zeros(1)
        rc = _lib.load().tmx_probe_fp64(self._h, int(kind), _lib.ptr(v))
        _lib.check(self._h, rc, "tmx_probe_fp64")
        return float(v[0])

    BATCH_HOST, BATCH_GRAPH = 0, 1

    def set_batch_mode(self, mode):
        """How batches drive the order loop (tmx_set_batch_mode): BATCH_HOST
        (the host issues order groups and forms block rounds) or BATCH_GRAPH
        (one CUDA graph runs the loop and its rounds on the device)."""
        rc = _lib.load().tmx_set_batch_mode(self._h, int(mode))
        _lib.check(self._h, rc, "tmx_set_batch_mode")

    @property
    def last_batch_mode(self):
        """The mode that computed the last batch (a graph-mode batch the
        graph does not cover runs in the host mode)."""
        v = np.zeros(1, np.int32)
        rc = _lib.load().tmx_last_batch_mode(self._h, _lib.iptr(v))
        _lib.check(self._h, rc, "tmx_last_batch_mode")
        return int(v[0])

    def profile(self, on=True):
        """Switch the per-kernel CUDA-event profile on or off
        (tmx_profile_enable); resets its counters and the timeline."""
        rc = _lib.load().tmx_profile_enable(self._h, int(bool(on)))
        _lib.check(self._h, rc, "tmx_profile_enable")

    TIMELINE_DTYPE = np.dtype([("kind", np.int32), ("stream", np.int32),
                               ("items", np.int32), ("start_ms", np.float64),
                               ("end_ms", np.float64)])

    def timeline(self):
        """Launch timeline since profile(True) (tmx_profile_timeline): one
        record per profiled launch or mark, times in ms."""
        lib = _lib.load()
        cnt = np.zeros(1, np.int64)
        rc = lib.tmx_profile_timeline(self._h, 0, None, _lib.lptr(cnt))
        _lib.check(self._h, rc, "tmx_profile_timeline")
        rec = np.zeros((int(cnt[0]), 5))
        rc = lib.tmx_profile_timeline(self._h, rec.shape[0], _lib.ptr(rec),
                                      _lib.lptr(cnt))
        _lib.check(self._h, rc, "tmx_profile_timeline")
        out = np.zeros(rec.shape[0], self.TIMELINE_DTYPE)
        for i, name in enumerate(self.TIMELINE_DTYPE.names):
            out[name] = rec[:, i]
        return out

    def tmatrix_batch(self, r_ev, wavelength, m, axis_ratio, min_order=10,
                      max_order=100, gauss_legendre_factor=2, tolerance=1e-4,
                      bessel_start=0):
        """Converged T-matrices of independent grains (SI units)."""
        r_ev = np.ascontiguousarray(r_ev, np.float64).ravel()
        n = r_ev.size
        wl = np.ascontiguousarray(np.broadcast_to(wavelength, (n,)), np.float64)
        mm = np.broadcast_to(np.asarray(m, np.complex128), (n,))
        mr = np.ascontiguousarray(mm.real)
        mi = np.ascontiguousarray(mm.imag)
        d = np.ascontiguousarray(np.broadcast_to(axis_ratio, (n,)), np.float64)
        sched = _lib.TmxSchedule(int(min_order), int(max_order),
                                 int(gauss_legendre_factor), int(bessel_start),
                                 float(tolerance))
        lib = _lib.load()
        with self._lock:
            rc = lib.tmx_tmatrix_batch(self._h, n, _lib.ptr(r_ev), _lib.ptr(wl),
                                       _lib.ptr(mr), _lib.ptr(mi), _lib.ptr(d),
                                       ctypes.byref(sched))
            _lib.check(self._h, rc, "tmx_tmatrix_batch")
            return self._results(n)


    def tmatrix_batch_fixed(self, r_ev, wavelength, m, axis_ratio, nmax, ngauss):
        """All m blocks of each grain at a given (nmax, ngauss), without the
        convergence loop."""
        r_ev = np.ascontiguousarray(r_ev, np.float64).ravel()
        n = r_ev.size
        wl = np.ascontiguousarray(np.broadcast_to(wavelength, (n,)), np.float64)
        mm = np.broadcast_to(np.asarray(m, np.complex128), (n,))
        mr = np.ascontiguousarray(mm.real)
        mi = np.ascontiguousarray(mm.imag)
        d = np.ascontiguousarray(np.broadcast_to(axis_ratio, (n,)), np.float64)
        nm = np.ascontiguousarray(np.broadcast_to(nmax, (n,)), np.int32)
        ng = np.ascontiguousarray(np.broadcast_to(ngauss, (n,)), np.int32)
        lib = _lib.load()
        with self._lock:
            rc = lib.tmx_tmatrix_batch_fixed(self._h, n, _lib.ptr(r_ev), _lib.ptr(wl),
                                             _lib.ptr(mr), _lib.ptr(mi), _lib.ptr(d),
                                             _lib.iptr(nm), _lib.iptr(ng))
            _lib.check(self._h, rc, "tmx_tmatrix_batch_fixed")
            return self._results(n)

    # block-kernel families (tmx_block_family) and the largest class size of
    # each dispatch bucket
    FAMILIES = ("warp_dfma", "warp_dmma", "cta32", "cta64", "cta")
    BUCKET_TOP = (8, 16, 32, 64, 128)

    def get_dispatch(self):
        """Block-kernel family of each class-size bucket (<= 8, 9..16,
        17..32, 33..64, 65..128) as an int32 array of 5."""
        out = np.zeros(5, np.int32)
        rc = _lib.load().tmx_get_dispatch(self._h, _lib.iptr(out))
        _lib.check(self._h, rc, "tmx_get_dispatch")
        return out

    def set_dispatch(self, families):
        fam = np.ascontiguousarray(families, np.int32).ravel()
        if fam.size != 5:
            raise ValueError("one family per bucket (5)")
        with self._lock:
            rc = _lib.load().tmx_set_dispatch(self._h, _lib.iptr(fam))
            _lib.check(self._h, rc, "tmx_set_dispatch")

    def autotune(self, r_ev, wavelength, m, axis_ratio, nmax, ngauss, reps=3):
        """Time every block-kernel family on the given grains at fixed orders
        and keep the fastest per bucket. Returns (table, ms) with ms[bucket,
        family] the median milliseconds per batch (-1: not run)."""
        r_ev = np.ascontiguousarray(r_ev, np.float64).ravel()
        n = r_ev.size
        wl = np.ascontiguousarray(np.broadcast_to(wavelength, (n,)), np.float64)
        mm = np.broadcast_to(np.asarray(m, np.complex128), (n,))
        mr = np.ascontiguousarray(mm.real)
        mi = np.ascontiguousarray(mm.imag)
        d = np.ascontiguousarray(np.broadcast_to(axis_ratio, (n,)), np.float64)
        nm = np.ascontiguousarray(np.broadcast_to(nmax, (n,)), np.int32)
        ng = np.ascontiguousarray(np.broadcast_to(ngauss, (n,)), np.int32)
        ms = np.zeros((5, 5), np.float64)
        lib = _lib.load()
        with self._lock:
            rc = lib.tmx_autotune(self._h, n, _lib.ptr(r_ev), _lib.ptr(wl),
                                  _lib.ptr(mr), _lib.ptr(mi), _lib.ptr(d),
                                  _lib.iptr(nm), _lib.iptr(ng), int(reps),
                                  _lib.ptr(ms))
            self._batch_id = self.batch_id + 1  # the last tuning batch is current
            _lib.check(self._h, rc, "tmx_autotune")
        return self.get_dispatch(), ms

    def tmatrix_batch_calculator(self, r_ev, wavelength, m, axis_ratio,
                                 maximum_order=200, tolerance=1e-4,
                                 gauss_legendre_factor=2, maximum_ngauss=500):
        """Converged T-matrices on the plain path's schedule (order loop, then
        quadrature loop; TMatrixCalculator::calculate_TMatrix)."""
        r_ev = np.ascontiguousarray(r_ev, np.float64).ravel()
        n = r_ev.size
        wl = np.ascontiguousarray(np.broadcast_to(wavelength, (n,)), np.float64)
        mm = np.broadcast_to(np.asarray(m, np.complex128), (n,))
        mr = np.ascontiguousarray(mm.real)
        mi = np.ascontiguousarray(mm.imag)
        d = np.ascontiguousarray(np.broadcast_to(axis_ratio, (n,)), np.float64)
        lib = _lib.load()
        with self._lock:
            rc = lib.tmx_tmatrix_batch_calculator(
                self._h, n, _lib.ptr(r_ev), _lib.ptr(wl), _lib.ptr(mr), _lib.ptr(mi),
                _lib.ptr(d), int(maximum_order), float(tolerance),
                int(gauss_legendre_factor), int(maximum_ngauss))
            _lib.check(self._h, rc, "tmx_tmatrix_batch_calculator")
            return self._results(n)

    def orientation_average(self, coefficient_sets, coef_set):
        """Replace the last batch's T-matrices by orientation averages:
        coef_set[i] indexes a row of coefficient_sets, -1 keeps grain i."""
        c = np.ascontiguousarray(np.atleast_2d(coefficient_sets), np.float64)
        idx = np.ascontiguousarray(coef_set, np.int32)
        lib = _lib.load()
        with self._lock:
            rc = lib.tmx_batch_orientation_average(self._h, _lib.ptr(c), c.shape[0],
                                                   c.shape[1], _lib.iptr(idx))
            self._batch_id = self.batch_id + 1
            _lib.check(self._h, rc, "tmx_batch_orientation_average")

    @staticmethod
    def _jobs(grain, *angles):
        arrs = np.broadcast_arrays(np.asarray(grain, np.int64),
                                   *[np.asarray(a, np.float64) for a in angles])
        shape = arrs[0].shape
        return shape, [np.ascontiguousarray(a.ravel()) for a in arrs]

    def scattering_matrix(self, grain, theta_in, phi_in, theta_out, phi_out,
                          alpha=0.0, beta=0.0):
        """Z (..., 4, 4) for lab-frame directions at particle orientation
        (alpha, beta); arguments broadcast against each other."""
        shape, (g, a, b, ti, pi, to, po) = self._jobs(grain, alpha, beta, theta_in,
                                                       phi_in, theta_out, phi_out)
        Z = np.zeros((g.size, 16))
        lib = _lib.load()
        with self._lock:
            rc = lib.tmx_batch_scattering_matrix(self._h, g.size, _lib.lptr(g),
                                                 _lib.ptr(a), _lib.ptr(b), _lib.ptr(ti),
                                                 _lib.ptr(pi), _lib.ptr(to),
                                                 _lib.ptr(po), _lib.ptr(Z), None)
            _lib.check(self._h, rc, "tmx_batch_scattering_matrix")
        return Z.reshape(shape + (4, 4))

    def extinction_matrix(self, grain, theta, phi, alpha=0.0, beta=0.0):
        """K (..., 4, 4) for the lab-frame direction (theta, phi)."""
        shape, (g, a, b, t, p) = self._jobs(grain, alpha, beta, theta, phi)
        K = np.zeros((g.size, 16))
        lib = _lib.load()
        with self._lock:
            rc = lib.tmx_batch_extinction_matrix(self._h, g.size, _lib.lptr(g),
                                                 _lib.ptr(a), _lib.ptr(b), _lib.ptr(t),
                                                 _lib.ptr(p), _lib.ptr(K))
            _lib.check(self._h, rc, "tmx_batch_extinction_matrix")
        return K.reshape(shape + (4, 4))

    def absorption_cross_sections(self, grain, theta, ngauss=100):
        """(ntheta, 2) array of (Cabs, Cabspol) of one grain."""
        th = np.ascontiguousarray(np.atleast_1d(theta), np.float64)
        out = np.zeros((th.size, 2))
        lib = _lib.load()
        with self._lock:
            rc = lib.tmx_batch_absorption_cross_sections(self._h, int(grain), th.size,
                                                         _lib.ptr(th), int(ngauss),
                                                         _lib.ptr(out))
            _lib.check(self._h, rc, "tmx_batch_absorption_cross_sections")
        return out

    def average_absorption_cross_section(self, grain, ngauss=20):
        out = np.zeros(1)
        lib = _lib.load()
        with self._lock:
            rc = lib.tmx_batch_average_absorption_cross_section(self._h, int(grain),
                                                                int(ngauss),
                                                                _lib.ptr(out))
            _lib.check(self._h, rc, "tmx_batch_average_absorption_cross_section")
        return float(out[0])

    def stream_tmatrices(self, capacity):
        """Stream the T-matrices of every following batch into a page-locked
        host buffer of `capacity` complex elements while the batch runs (each
        block round copies its range as soon as it is done); 0 stops."""
        lib = _lib.load()
        with self._lock:
            rc = lib.tmx_set_tmatrix_sink(self._h, None, 0)
            _lib.check(self._h, rc, "tmx_set_tmatrix_sink")
            if getattr(self, "_sink", None):
                lib.tmx_host_free(self._sink[0])
                self._sink = None
            if capacity <= 0:
                return
            ptr = lib.tmx_host_alloc(16 * int(capacity))
            if not ptr:
                raise _lib.TmxError("page-locked allocation of %d bytes failed"
                                    % (16 * int(capacity)))
            rc = lib.tmx_set_tmatrix_sink(
                self._h, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)),
                int(capacity))
            if rc != 0:
                lib.tmx_host_free(ptr)
            _lib.check(self._h, rc, "tmx_set_tmatrix_sink")
            self._sink = (ptr, int(capacity))

    def tmatrices(self):
        """Every T-matrix of the last batch in one transfer: (flat complex
        array, offsets) with grain i's T-matrix at flat[offsets[i]:] in the
        reference block layout (offsets[i] = -1: none). With a stream buffer
        (stream_tmatrices) the array is a view of it that the next batch
        overwrites, and only what was not streamed yet is copied."""
        lib = _lib.load()
        n = self._last_n()
        total = ctypes.c_int64()
        offsets = np.zeros(n, np.int64)
        with self._lock:
            rc = lib.tmx_batch_tmatrix_total(self._h, ctypes.byref(total))
            _lib.check(self._h, rc, "tmx_batch_tmatrix_total")
            total = total.value
            sink = getattr(self, "_sink", None)
            if sink and sink[1] >= total:
                buf = (ctypes.c_char * (16 * max(1, total))).from_address(sink[0])
                flat = np.frombuffer(buf, dtype=np.complex128, count=total)
                dst = ctypes.cast(sink[0], ctypes.POINTER(ctypes.c_double))
            else:
                flat = self._pinned.array((2 * max(1, total),)).view(np.complex128)[:total]
                dst = flat.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            rc = lib.tmx_batch_tmatrices(self._h, dst, _lib.lptr(offsets))
            _lib.check(self._h, rc, "tmx_batch_tmatrices")
        return flat, offsets

    @property
    def batch_id(self):
        """Counter of the batches (and T-matrix replacements) of this
        context: results of an earlier id are gone."""
        return getattr(self, "_batch_id", 0)

    def _results(self, n):
        self._n = n
        self._batch_id = self.batch_id + 1
        lib = _lib.load()
        nmax = np.zeros(n, np.int32)
        ngauss = np.zeros(n, np.int32)
        status = np.zeros(n, np.int32)
        q = np.zeros((n, 6))
        rc = lib.tmx_batch_results(self._h, _lib.iptr(nmax), _lib.iptr(ngauss),
                                   _lib.iptr(status), _lib.ptr(q))
        _lib.check(self._h, rc, "tmx_batch_results")
        return BatchResult(self, n, nmax, ngauss, status, q)

    def observables(self, thetas, coefficients=None):
        """(n, ntheta, 3) array of (Qext, Qextpol, Qextcpol) of the last batch,
        orientation-averaged with the given expansion coefficients."""
        th = np.ascontiguousarray(np.atleast_1d(thetas), np.float64)
        c = None if coefficients is None else np.ascontiguousarray(coefficients, np.float64)
        lib = _lib.load()
        n = self._last_n()
        q = self._pinned.array((n, len(th), 3))
        with self._lock:
            rc = lib.tmx_batch_observables(self._h, len(th), _lib.ptr(th),
                                           None if c is None else _lib.ptr(c),
                                           0 if c is None else len(c), _lib.ptr(q))
            _lib.check(self._h, rc, "tmx_batch_observables")
        return q

    def gradients(self, thetas, coefficients=None):
        """(q, dq): q as observables(); dq (n, ntheta, 3, 4) derivatives with
        respect to (Re m, Im m, r_ev, axis ratio) at the batch's orders."""
        th = np.ascontiguousarray(np.atleast_1d(thetas), np.float64)
        c = None if coefficients is None else np.ascontiguousarray(coefficients, np.float64)
        lib = _lib.load()
        n = self._last_n()
        q = self._pinned.array((n, len(th), 3))
        dq = self._pinned.array((n, len(th), 3, 4))
        with self._lock:
            rc = lib.tmx_batch_gradients(self._h, len(th), _lib.ptr(th),
                                         None if c is None else _lib.ptr(c),
                                         0 if c is None else len(c), _lib.ptr(q),
                                         _lib.ptr(dq))
            _lib.check(self._h, rc, "tmx_batch_gradients")
        return q, dq

    def _last_n(self):
        if getattr(self, "_n", None) is None:
            raise _lib.TmxError("no batch has been computed")
        return self._n


_default = None


def default_context():
    global _default
    if _default is None:
        _default = Context(0)
    return _default
