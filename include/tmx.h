/* tmx.h -- C ABI of the B200 T-matrix library (libtmx.so).
 *
 * The library computes EBCM T-matrices of spheroids and their orientation-
 * and shape-averaged observables on one NVIDIA B200 (sm_100a) in FP64. It is
 * the drop-in replacement of the CosTuuM T-matrix path: the host drivers
 * (CosTuuM's TaskManager + QuickSched, src/TaskManager.hpp:445-1346, and its
 * Python module, src/CTMModule.cpp:146-478) bind these entry points instead
 * of building and running a task graph on host threads.
 *
 * Conventions
 *   - plain pointers and sizes only; every array argument is host memory
 *     unless its name ends in _dev;
 *   - complex numbers are interleaved (re, im) doubles;
 *   - T-matrices use the reference's block layout (TMatrixResource,
 *     src/TMatrixResource.hpp:195-213): block m (m = 0..nmax) is a
 *     2nb x 2nb row-major complex matrix, nb = nmax for m = 0 and
 *     nmax + 1 - m otherwise; row (i, n) sits at i * nb + n - max(m, 1);
 *     blocks follow each other in m order (tmx_tmatrix_size());
 *   - functions return TMX_OK (0) or a negative tmx_error; per-grain
 *     outcomes are reported as status bits, never by aborting (the reference
 *     calls abort() on non-convergence in its plain path).
 */
#ifndef TMX_H
#define TMX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tmx_ctx tmx_ctx;

enum tmx_error {
  TMX_OK = 0,
  TMX_ERR_INVALID = -1,  /* bad argument; see tmx_last_error() */
  TMX_ERR_CUDA = -2,     /* a CUDA call failed */
  TMX_ERR_NOMEM = -3,    /* device allocation failed */
  TMX_ERR_STATE = -4,    /* no batch computed yet / index out of range */
  TMX_ERR_NO_DEVICE = -5 /* no usable CUDA device */
};

/* per-grain status bits */
enum tmx_grain_status {
  TMX_GRAIN_OK = 0,
  TMX_GRAIN_NOT_CONVERGED = 1, /* reached maximum_order - 1 (reference:
                                  silent in the task path) */
  TMX_GRAIN_SINGULAR = 2,      /* zero pivot in a Q block */
  TMX_GRAIN_NAN = 4,           /* non-finite sums */
  TMX_GRAIN_BAD_INPUT = 8,     /* r_ev, wavelength or axis ratio <= 0 */
  TMX_GRAIN_TOO_LARGE = 16     /* block larger than the on-chip solver */
};

/* Convergence schedule of the task-based path (TaskManager(min_order,
 * max_order, gauss_legendre_factor, tolerance), src/TaskManager.hpp:371):
 * orders min_order .. max_order - 1 with ngauss = factor * order, stop at the
 * first order whose m = 0 Qsca and Qext both change by <= tolerance. */
typedef struct tmx_schedule {
  int32_t min_order;             /* default 10 */
  int32_t max_order;             /* default 100 (exclusive) */
  int32_t gauss_legendre_factor; /* default 2 */
  int32_t bessel_start;          /* start index of the downward j_n ratio
                                    recurrence: 0 = automatic,
                                    max(nmax, |z|) + 48 capped at 800 (same
                                    doubles as the reference's fixed start
                                    SPECIALFUNCTIONS_BESSEL_NMAX = 800);
                                    > 0 = that fixed start */
  double tolerance;              /* default 1e-4 */
} tmx_schedule;

/* Create a context on CUDA device `device` (the context owns a stream,
 * device buffers and cached quadrature/Wigner tables). Replaces the
 * QuickSched object + TMatrixAuxiliarySpaceManager of the reference
 * (src/QuickSchedWrapper.hpp:302, src/TMatrixResource.hpp:376-435). */
int tmx_create(tmx_ctx **ctx, int device);
void tmx_destroy(tmx_ctx *ctx);
const char *tmx_last_error(const tmx_ctx *ctx);

/* Complex elements of a T-matrix with all m blocks up to nmax. */
int64_t tmx_tmatrix_size(int32_t nmax);

/* Converged T-matrices of n independent grains (the InteractionTask ->
 * TMatrixM0Task convergence chain of TaskManager.hpp:1146-1197 followed by
 * TMatrixMAllTask for every m, :1313-1327). Inputs are host arrays of length
 * n: equal-volume radius and wavelength in metres, refractive index
 * (mr + i mi), axis ratio d = a/b. The results stay on the device until the
 * next batch; read them with tmx_batch_results / tmx_batch_tmatrix. */
int tmx_tmatrix_batch(tmx_ctx *ctx, int64_t n, const double *r_ev,
                      const double *wavelength, const double *mr,
                      const double *mi, const double *axis_ratio,
                      const tmx_schedule *schedule);

/* The same computation in two steps: upload the inputs (host -> device),
 * then compute from device-resident inputs (may be repeated). */
int tmx_batch_upload(tmx_ctx *ctx, int64_t n, const double *r_ev,
                     const double *wavelength, const double *mr,
                     const double *mi, const double *axis_ratio,
                     const tmx_schedule *schedule);
int tmx_batch_compute(tmx_ctx *ctx);

/* The block computation of a batch at given orders, without the convergence
 * loop: grain i gets all m blocks at (nmax[i], ngauss[i]) (the state of a
 * TMatrixMAllTask run after ConvergedSizeResources fixed the order,
 * src/TMatrixResource.hpp:893-1120, plus its m = 0 block). For finite
 * differences and gradients at a fixed order. */
int tmx_tmatrix_batch_fixed(tmx_ctx *ctx, int64_t n, const double *r_ev,
                            const double *wavelength, const double *mr,
                            const double *mi, const double *axis_ratio,
                            const int32_t *nmax, const int32_t *ngauss);

/* Converged T-matrices on the plain path's schedule
 * (TMatrixCalculator::calculate_TMatrix, src/TMatrixCalculator.hpp:64-213,
 * which the reference runs one grain at a time): starting at
 * nmax = int(max(4, x + 4.05 x^(1/3))), raise nmax until the m = 0 Qsca and
 * Qext change by <= tolerance (ngauss = ndgs nmax), then raise ngauss from
 * ndgs nmax + 1 until they change by <= tolerance; then every m block at the
 * final (nmax, ngauss). r_ev is the equal-volume radius. A grain that reaches
 * maximum_order or maximum_ngauss (the reference aborts) gets
 * TMX_GRAIN_NOT_CONVERGED and keeps its last order. The m = 0 steps run to
 * order 255; a grain whose final order is above 128 (the block kernels'
 * class limit; in practice a grain that ran to maximum_order 200 without
 * converging) also gets TMX_GRAIN_TOO_LARGE and no T-matrix (nmax 0).
 * Results as for tmx_tmatrix_batch;
 * q[6 i + 0], q[6 i + 1] hold the m = 0 sums of the last step and
 * q[6 i + 4], q[6 i + 5] their relative changes. */
int tmx_tmatrix_batch_calculator(tmx_ctx *ctx, int64_t n, const double *r_ev,
                                 const double *wavelength, const double *mr,
                                 const double *mi, const double *axis_ratio,
                                 int32_t maximum_order, double tolerance,
                                 int32_t ndgs, int32_t maximum_ngauss);

/* Per-grain results of the last batch (any pointer may be NULL):
 * nmax, ngauss, status bits, and q[6 * i + {0..5}] =
 * {m=0 Qsca, m=0 Qext of the converged order, full Qsca, full Qext
 *  (TMatrixQTask, src/TMatrixResource.hpp:1136-1210), dQs, dQe}.
 * Qsca/Qext are the reference's unnormalised sums. */
int tmx_batch_results(tmx_ctx *ctx, int32_t *nmax, int32_t *ngauss,
                      int32_t *status, double *q);

/* Copy the T-matrix of grain `grain` of the last batch into `out`
 * (2 * tmx_tmatrix_size(nmax) doubles). */
int tmx_batch_tmatrix(tmx_ctx *ctx, int64_t grain, double *out);

/* Every T-matrix of the last batch in one transfer: the reference keeps one
 * TMatrixResource per grain (src/TMatrixResource.hpp:60-276) that its
 * callers read in place; here they sit in one ragged device buffer.
 * *total = complex elements of that buffer. tmx_batch_tmatrices copies it
 * into out (2 * total doubles, may be NULL) and writes offsets[i] (may be
 * NULL) = complex offset of grain i's T-matrix in out (tmx_tmatrix_size(
 * nmax[i]) elements in the block layout above), -1 for a grain without
 * one. When out is the sink set below, only the part that the block rounds
 * have not already streamed is copied. */
int tmx_batch_tmatrix_total(tmx_ctx *ctx, int64_t *total);
int tmx_batch_tmatrices(tmx_ctx *ctx, double *out, int64_t *offsets);

/* Stream the T-matrices of every following batch into page-locked host
 * memory (tmx_host_alloc or cudaHostRegister; capacity in complex
 * elements): each block round copies its range as soon as its blocks are
 * done, overlapping the rest of the batch, at the offsets that
 * tmx_batch_tmatrices reports; ranges beyond the capacity are left to
 * tmx_batch_tmatrices. The buffer is rewritten by every batch. host = NULL
 * stops streaming. TMX_ERR_INVALID if host is not page-locked. */
int tmx_set_tmatrix_sink(tmx_ctx *ctx, double *host, int64_t capacity);

/* Measured FP64 throughput of this device in TFLOP/s: kind 0 = DFMA pipe,
 * kind 1 = DMMA tensor pipe (mma.sync m8n8k4 f64). */
int tmx_probe_fp64(tmx_ctx *ctx, int kind, double *tflops);

/* CUDA-event timer on the library's stream (the stream every kernel of the
 * context is launched on). */
int tmx_timer_start(tmx_ctx *ctx);
int tmx_timer_stop(tmx_ctx *ctx, double *ms);

/* Per-kernel device time: when enabled, every launch of the kernels below
 * is bracketed by CUDA events on the stream it runs on; tmx_profile_read
 * returns the summed milliseconds, the launch count and the FP64 flops
 * (blocks: executed flops of the parity-class algorithm; orientation
 * average and amplitudes: the flops of their index spaces), and
 * tmx_profile_bytes the algorithmic bytes (each operand read or written
 * once: T-matrices in and out of the orientation average, averaged
 * T-matrices in and amplitudes out, the shape average's inputs, weights and
 * outputs). Enabling resets the counters. */
enum tmx_profile_kernel {
  TMX_PROF_BLOCKS = 0,    /* block kernels: assembly + LU + solve */
  TMX_PROF_TABLES = 1,    /* node scalars and Bessel tables */
  TMX_PROF_ORIENT = 2,    /* orientation average (AlignmentAverageTask) */
  TMX_PROF_AMP = 3,       /* scattering amplitudes (Extinction/Absorption/
                             ScatteringMatrixTask) */
  TMX_PROF_SHAPE_AVG = 4, /* shape average (ShapeAveragingTask) */
  TMX_PROF_TANGENTS = 5,  /* tangent kernels of tmx_batch_gradients */
  TMX_PROF_KERNELS = 6
};
int tmx_profile_enable(tmx_ctx *ctx, int on);
int tmx_profile_read(tmx_ctx *ctx, int kernel, double *ms, int64_t *launches,
                     double *flops);
int tmx_profile_bytes(tmx_ctx *ctx, int kernel, double *bytes);

/* Timeline of the profiled launches since tmx_profile_enable (the device-side
 * counterpart of the reference's per-task log, QuickSched's task output):
 * 5 doubles per record, {kind, stream, items, start_ms, end_ms}, times from
 * the enable call on the library stream. kind: a tmx_profile_kernel, or a
 * mark (start == end) below; stream: 0 the library stream (convergence
 * loop), 1 and 2 the block-round streams, 3..8 their bucket streams; items:
 * work items of a block launch. At most cap records are written; *count
 * receives the number available. */
enum tmx_timeline_mark {
  TMX_TL_BATCH_START = -1, /* tmx_batch_compute's first launch */
  TMX_TL_LOOP_END = -2,    /* the order loop's last launch has finished */
  TMX_TL_BATCH_END = -3    /* every launch of the batch has finished */
};
int tmx_profile_timeline(tmx_ctx *ctx, int64_t cap, double *records,
                         int64_t *count);

/* How tmx_batch_compute drives the order loop.
 * TMX_BATCH_HOST: the host issues the order groups one ahead of the GPU,
 * reads each group's outcome and forms the block rounds (the default).
 * TMX_BATCH_GRAPH: one CUDA graph per batch shape whose conditional WHILE
 * node runs the whole loop on the device -- order steps, convergence,
 * rounds of the grains that became final, Q sums -- until no grain is left;
 * the host only uploads the batch and reads the results (QuickSched's role,
 * TaskManager.hpp:1146-1197 and :1313-1327, played by the device). Results
 * are bit-identical to the host mode. Batches the graph mode does not cover
 * (maximum_order above 101, tables beyond 24 GB, profiling or autotuning on)
 * and a batch whose T-matrix or LU storage outgrows the estimate run in the
 * host mode. */
enum tmx_batch_mode { TMX_BATCH_HOST = 0, TMX_BATCH_GRAPH = 1 };
int tmx_set_batch_mode(tmx_ctx *ctx, int mode);
int tmx_get_batch_mode(tmx_ctx *ctx, int *mode);
/* Which mode computed the last batch (TMX_BATCH_HOST or TMX_BATCH_GRAPH). */
int tmx_last_batch_mode(tmx_ctx *ctx, int *mode);

/* Host-side times of the last tmx_batch_compute, out[4] in ms: wall time of
 * the call, time blocked on the order loop's events and the final
 * synchronisation, host set-up of the block rounds, and (out[3]) the number
 * of order groups the loop waited for. Always recorded. */
int tmx_batch_host_times(tmx_ctx *ctx, double *out);

/* FP64 flops of the last batch counted with the unreduced per-grain model
 * (every chain order and every m block as a full 2nb x 2nb LU + solve);
 * counted only for batches computed while profiling is enabled, else 0. */
double tmx_batch_flops_survey(const tmx_ctx *ctx);

/* ------------------------------------------------ block-kernel dispatch ---
 *
 * The class items of a block round are launched in buckets by class size nb:
 * bucket 0 nb <= 8, 1 nb 9..16, 2 nb 17..32, 3 nb 33..64, 4 nb 65..128. Each
 * bucket runs one kernel family; a family can run a bucket when its capacity
 * covers the bucket's sizes. The table applies to every block launch of the
 * context (batched, fixed-order and calculator schedules, gradients);
 * tmx_tmatrix_fixed_noalloc keeps the default. Families compute the same
 * sums in different orders, so results differ in the last bits between
 * tables. */
enum tmx_block_family {
  TMX_FAMILY_WARP_DFMA = 0, /* one warp per item, DFMA register tiles; nb <= 8 */
  TMX_FAMILY_WARP_DMMA = 1, /* one warp per item, DMMA m8n8k4 tiles; nb <= 16 */
  TMX_FAMILY_CTA32 = 2,     /* four warps per item; nb <= 32 */
  TMX_FAMILY_CTA64 = 3,     /* eight warps per item; nb <= 64 */
  TMX_FAMILY_CTA = 4        /* 256 threads per item, 4x4 tiles; nb <= 128 */
};
#define TMX_DISPATCH_BUCKETS 5
#define TMX_DISPATCH_FAMILIES 5

/* Page-locked host memory (cudaMallocHost) for result arrays: device to
 * host copies into it run as direct DMA instead of through the driver's
 * staging buffers. NULL on failure; release with tmx_host_free. */
void *tmx_host_alloc(size_t bytes);
void tmx_host_free(void *p);

/* family[5]: the family of each bucket (default 0, 1, 2, 3, 4). */
int tmx_get_dispatch(const tmx_ctx *ctx, int32_t *family);
/* Sets the family of each bucket; TMX_ERR_INVALID (table unchanged) if a
 * family cannot run its bucket. */
int tmx_set_dispatch(tmx_ctx *ctx, const int32_t *family);

/* Autotuner for the dispatch table: computes the given grains at fixed
 * orders (as tmx_tmatrix_batch_fixed) reps times with each family in every
 * bucket it can run, the buckets' launches serialised on the library stream
 * and timed with CUDA events, then moves each bucket that the sample reaches
 * to the family with the smallest median time if that is at least 5 % below
 * the median of its current family (else the bucket keeps its family).
 * ms (may be NULL) receives [bucket][family] median milliseconds per batch,
 * -1 where the family cannot run the bucket or the sample has no item of
 * that size. Afterwards the last tuning batch is the current batch. */
int tmx_autotune(tmx_ctx *ctx, int64_t n, const double *r_ev,
                 const double *wavelength, const double *mr, const double *mi,
                 const double *axis_ratio, const int32_t *nmax,
                 const int32_t *ngauss, int reps, double *ms);

/* ------------------------------------------------ averaged observables ---
 *
 * Orientation distribution expansion coefficients p_0 .. p_order
 * (OrientationDistribution::initialise, src/OrientationDistribution.hpp:
 * 220-243 and its subclasses): kind 0 random orientation (p(beta) = 1/2,
 * numerical quadrature), 1 Mishchenko (param = <cos^2 beta>,
 * src/MishchenkoOrientationDistribution.hpp:107-118), 2 Davis-Greenstein
 * perfect alignment (param = axis ratio,
 * src/DavisGreensteinOrientationDistribution.hpp:81-102), 3 custom p(beta)
 * given by fn(beta, arg) (src/PyOrientationDistribution.hpp:458-600). */
int tmx_orientation_coefficients(int kind, double param, int order,
                                 double (*fn)(double, void *), void *arg,
                                 double *out);

/* Shape distribution quadrature nodes and weights (ShapeDistribution::
 * evaluate, src/ShapeDistribution.hpp:95-106): kind 0 the default
 * distribution on [0.5, 1.5], kind 1 Draine & Hensley
 * (src/DraineHensleyShapeDistribution.hpp; param1 = cutoff, param2 =
 * fraction, as its constructor). limits (may be NULL) receives the minimum
 * and maximum axis ratio. */
int tmx_shape_distribution(int kind, int npoints, double param1, double param2,
                           double *shapes, double *weights, double *limits);

/* R_V / R_S, the ratio of the equal-volume and equal-surface-area sphere
 * radii of a spheroid with axis ratio d
 * (src/SpecialFunctions.hpp:557-583; CTMModule.cpp:66-95). */
double tmx_rv_over_rs(double axis_ratio);

enum tmx_table_flags {
  TMX_TABLE_ABSORPTION = 1,
  TMX_TABLE_EXTINCTION = 2,
  TMX_TABLE_SCATTERING = 4,
  TMX_TABLE_ACCOUNT_FOR_SCATTERING = 8
};

/* The get_table computation (src/CTMModule.cpp:146-478 with the task graph of
 * src/TaskManager.hpp:445-1346) for a grid of compositions x sizes x
 * wavelengths x shapes. sizes and lambdas must already be sorted ascending
 * (the reference sorts them). mr/mi[(type * nsizes + size) * nlambda + l] is
 * the refractive index of each cell; orient_set[size * nshape + shape] picks a
 * row of coeffs[nsets][ncoef] (or -1: no orientation averaging); ncoef must
 * exceed 2 nmax. Outputs (host): out_q[cell][theta][k] with k = (Qabs,
 * Qabspol) if TMX_TABLE_ABSORPTION then (Qext, Qextpol, Qextcpol) if
 * TMX_TABLE_EXTINCTION; out_z[cell][theta][phi][4][4] on the reference's
 * scattering grid (theta_in = pi/2, ntheta Gauss-Legendre zenith angles,
 * 2 ntheta Gauss-Legendre azimuths); grain_status[cell][shape] (may be
 * NULL). ngauss is number_of_quadrature_angles of the scattering
 * subtraction. */
int tmx_get_table(tmx_ctx *ctx, int32_t ntypes, int32_t nsizes,
                  const double *sizes, int32_t nlambda, const double *lambdas,
                  int32_t ntheta, const double *thetas, int32_t nshape,
                  const double *shapes, const double *shape_weights,
                  const double *mr, const double *mi, const int32_t *orient_set,
                  int32_t nsets, const double *coeffs, int32_t ncoef,
                  int32_t flags, int32_t ngauss, const tmx_schedule *schedule,
                  double *out_q, double *out_z, int32_t *grain_status);

/* Orientation-averaged extinction coefficients of every grain of the last
 * batch at the zenith angles thetas (ExtinctionCoefficientTask::execute,
 * src/ExtinctionCoefficientTask.hpp:626-653, on the AlignmentAverageTask
 * output): q[(grain * ntheta + t) * 3 + {0,1,2}] = {Qext, Qextpol,
 * Qextcpol}. Without the scattering subtraction the reference's Qabs and
 * Qabspol equal Qext and Qextpol. coeffs (ncoef >= 2 nmax + 1 values) are
 * the orientation distribution's expansion coefficients; NULL keeps the
 * particle-frame T-matrix. */
int tmx_batch_observables(tmx_ctx *ctx, int32_t ntheta, const double *thetas,
                          const double *coeffs, int32_t ncoef, double *q);

/* Derivatives of those coefficients at the orders of the last batch with
 * respect to (Re m, Im m, r_ev, axis ratio): dq[((grain * ntheta + t) * 3 +
 * k) * 4 + p]. Forward-mode through dT = -(dRgQ + T dQ) Q^-1 with the LU
 * factors of each block; no counterpart in the reference (which has no
 * derivatives). q (may be NULL) receives the coefficients themselves. */
int tmx_batch_gradients(tmx_ctx *ctx, int32_t ntheta, const double *thetas,
                        const double *coeffs, int32_t ncoef, double *q,
                        double *dq);

/* ------------------------------------------- plain-path observables ---
 *
 * The per-particle queries of the reference's TMatrix object
 * (src/PyTMatrix.hpp, src/TMatrix.hpp), for any grain of the last batch.
 *
 * Replace every grain's T-matrix by its orientation average
 * (TMatrixCalculator::apply_orientation_distribution,
 * src/TMatrixCalculator.hpp:229-307): coef_set[i] selects row coef_set[i] of
 * coeffs (nsets x ncoef expansion coefficients p_0..), -1 keeps grain i.
 * Gradients are unavailable afterwards. */
int tmx_batch_orientation_average(tmx_ctx *ctx, const double *coeffs,
                                  int32_t nsets, int32_t ncoef,
                                  const int32_t *coef_set);

/* Scattering matrices Z (row-major 4 x 4 per job) and, if S is not NULL,
 * the amplitude matrices S (2 x 2 complex per job) for incoming
 * (theta_in, phi_in) and outgoing (theta_out, phi_out) lab-frame directions
 * at a particle whose symmetry axis has azimuth alpha and zenith beta
 * (TMatrix::get_scattering_matrix, src/TMatrix.hpp:1891-1952, with the frame
 * rotation of :1306-1482). Angles in radians; grain[j] indexes the batch. */
int tmx_batch_scattering_matrix(tmx_ctx *ctx, int64_t njobs,
                                const int64_t *grain, const double *alpha,
                                const double *beta, const double *theta_in,
                                const double *phi_in, const double *theta_out,
                                const double *phi_out, double *Z, double *S);

/* Extinction matrices K (row-major 4 x 4 per job) for the direction
 * (theta, phi) (TMatrix::get_extinction_matrix, src/TMatrix.hpp:1972-2010). */
int tmx_batch_extinction_matrix(tmx_ctx *ctx, int64_t njobs,
                                const int64_t *grain, const double *alpha,
                                const double *beta, const double *theta,
                                const double *phi, double *K);

/* Absorption cross sections (Cabs, Cabspol) at zenith angles theta: the
 * forward-amplitude extinction minus the scattering integral over ngauss x
 * ngauss incoming directions (TMatrix::get_absorption_cross_sections,
 * src/TMatrix.hpp:2133-2225); out[2 t], out[2 t + 1]. */
int tmx_batch_absorption_cross_sections(tmx_ctx *ctx, int64_t grain,
                                        int32_t ntheta, const double *theta,
                                        int32_t ngauss, double *out);

/* Orientation-averaged absorption cross section: the Cabs of the ngauss
 * Gauss-Legendre zenith angles, weighted and halved
 * (TMatrix::get_average_absorption_cross_section, src/TMatrix.hpp:2260-2287). */
int tmx_batch_average_absorption_cross_section(tmx_ctx *ctx, int64_t grain,
                                               int32_t ngauss, double *out);

/* T-matrix of one grain at a fixed (nmax, ngauss), all m blocks, for callers
 * that cannot allocate device memory -- e.g. a host application whose device
 * memory is owned by another framework's caching allocator, or a per-call
 * path that cannot pay cudaMalloc/cudaFree's implicit synchronisation. No
 * counterpart in the reference. It calls no cudaMalloc/cudaFree: its
 * intermediates live in one static device array of 2.25 MiB that every GPU
 * loading the library keeps until exit. Limits: 2 <= nmax <= 32,
 * 1 <= ngauss <= 64 (larger sizes return TMX_ERR_INVALID with a message on
 * stderr). The caller passes the grain (SI units) and a device buffer T_dev
 * of 2 * tmx_tmatrix_size(nmax) doubles; the work is enqueued on `stream`
 * (a cudaStream_t, NULL = legacy default stream) and is complete when that
 * stream is. status_dev (a device int32_t, may be NULL) receives the grain's
 * status bits in stream order (tmx_grain_status: 0, or TMX_GRAIN_SINGULAR /
 * TMX_GRAIN_NAN when a class block had a zero pivot or non-finite entries);
 * the return value reports argument and CUDA errors only, so a caller that
 * passes NULL cannot tell a failed solve from a valid T-matrix. The first
 * call on a device looks up the array's device address with that device
 * current; make that first call before any stream capture. All calls share
 * the array: calls that overlap on the GPU race. */
int tmx_tmatrix_fixed_noalloc(double r_ev, double wavelength, double mr,
                              double mi, double axis_ratio, int32_t nmax,
                              int32_t ngauss, double *T_dev,
                              int32_t *status_dev, void *stream);

/* Number of this library's kernels launched since the context was created. */
int64_t tmx_kernel_launches(const tmx_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif /* TMX_H */
