// Table kernels: node scalars, spherical Bessel/Hankel tables and Wigner d
// tables on device (sm_100a, FP64).
//
// This translation unit is compiled with --fmad=false: the recurrences below
// follow the reference's operation order (src/SpecialFunctions.hpp) and, with
// no fused multiply-add, round the way the reference's x86-64 build rounds,
// except for the complex reciprocal of the downward j_n(m k r) recurrence
// (see bessel_j_complex).
// Transcendentals (sin, cos, cosh, sinh) come from CUDA's libdevice and may
// differ from the C library by an ulp.
#include <algorithm>

#include "tmx_common.cuh"
#include "tmx_kernels.h"

// ---------------------------------------------------------------- Bessel --

// Start index of the downward ratio recurrence. The reference starts at
// n = 800 for every argument (SPECIALFUNCTIONS_BESSEL_NMAX). Above
// max(nmax, |z|) the recurrence contracts errors by about (|z| / 2n)^2 per
// step, so a start 48 orders above max(nmax, |z|) reaches the same doubles
// as a start at 800 (tests/test_bessel_start.py checks this bit for bit).
// bessel_start > 0 forces a fixed start.
__device__ __forceinline__ int bessel_nstart(int bessel_start, int nmax,
                                             double absz) {
  if (bessel_start > 0) {
    return bessel_start;
  }
  const int hi = max(nmax, (int)ceil(absz)) + TMX_BESSEL_MARGIN;
  return min(hi, 800);
}

// Spherical j_n and [z j_n]'/z, n = 1..nmax, for a real argument, by the
// downward ratio recurrence rho_n = j_n / j_{n-1} started at n = nstart with
// rho ~ z / (2 nstart + 1), then j_n = rho_n j_{n-1} upward
// (SpecialFunctions::spherical_j_jdj_array, SpecialFunctions.hpp:201-240).
// The ratios go to rho[(n-1) * rs] (shared memory, or the output slots
// themselves); out[(n-1) * stride + {0, 1}] = (j_n, [z j_n]'/z), stored as
// one 16-byte pair.
__device__ static void bessel_j_real(int nmax, int nstart, double z,
                                     double *out, int stride, double *rho,
                                     int rs) {
  const double zinv = 1. / z;
  double cur = z / (2. * nstart + 1.);
  for (int index = nstart - 1; index >= 1; --index) {
    const double twoip1 = 2. * index + 1.;
    const double nxt = 1. / (twoip1 * zinv - cur);
    if (index - 1 < nmax) {
      rho[(index - 1) * rs] = nxt; // rho_{index-1} (0-based), kept
    }
    cur = nxt;
  }
  const double j0 = sin(z) * zinv;
  double jprev = rho[0] * j0;
  *reinterpret_cast<double2 *>(out) = make_double2(jprev, j0 - jprev * zinv);
  for (int i = 1; i < nmax; ++i) {
    const double ji = rho[i * rs] * jprev;
    const double ip1 = i + 1.;
    *reinterpret_cast<double2 *>(out + i * stride) =
        make_double2(ji, jprev - ip1 * zinv * ji);
    jprev = ji;
  }
}

// Spherical y_n and [z y_n]'/z by the upward recurrence from y_1, y_2
// (SpecialFunctions::spherical_y_ydy_array, SpecialFunctions.hpp:106-140).
__device__ static void bessel_y_real(int nmax, double z, double *out,
                                     int stride) {
  double sinz, cosz;
  sincos(z, &sinz, &cosz);
  const double zinv = 1. / z;
  const double zinv2 = zinv * zinv;
  const double zinv3 = zinv2 * zinv;
  double y0 = -cosz * zinv2 - sinz * zinv;
  double y1 = (-3. * zinv3 + zinv) * cosz - 3. * zinv2 * sinz;
  *reinterpret_cast<double2 *>(out) = make_double2(y0, -zinv * (cosz + y0));
  if (nmax > 1) {
    *reinterpret_cast<double2 *>(out + stride) =
        make_double2(y1, y0 - 2. * zinv * y1);
  }
  for (int i = 2; i < nmax; ++i) {
    const double twoip1 = 2. * i + 1.;
    const double ip1 = i + 1.;
    const double yi = twoip1 * zinv * y1 - y0;
    *reinterpret_cast<double2 *>(out + i * stride) =
        make_double2(yi, y1 - ip1 * zinv * yi);
    y0 = y1;
    y1 = yi;
  }
}

// complex sine sin(x) cosh(y) + i cos(x) sinh(y)
__device__ static cplx csin_dev(cplx z) {
  double s, c;
  sincos(z.x, &s, &c);
  return mkc(s * cosh(z.y), c * sinh(z.y));
}

// Complex-argument version of bessel_j_real: every constant enters as a
// complex number in the reference (std::complex arithmetic); multiplying by a
// complex number with zero imaginary part equals scaling by its real part
// bit for bit, which is what is done here. The reciprocal in the downward
// recurrence is conj(w) / |w|^2 (one real division; |w| ~ (2n + 1) / |z|
// is far from overflow and underflow), where the reference's complex
// division takes three (Smith's algorithm): the ratios agree to the last
// few bits.
// out[(n-1) * stride + {0,1,2,3}] = (Re j, Im j, Re dj, Im dj), stored as
// two 16-byte pairs; the ratios go to rho[(n-1) * rs].
__device__ static void bessel_j_complex(int nmax, int nstart, cplx z,
                                        double *out, int stride, cplx *rho,
                                        int rs) {
  const cplx zinv = cinv(z);
  cplx cur = cdiv(z, mkc(2. * nstart + 1., 0.));
  for (int index = nstart - 1; index >= 1; --index) {
    const double twoip1 = 2. * index + 1.;
    const cplx w = csub(cscale(zinv, twoip1), cur);
    const double inv = 1. / (w.x * w.x + w.y * w.y);
    const cplx nxt = mkc(w.x * inv, -w.y * inv);
    if (index - 1 < nmax) {
      rho[(index - 1) * rs] = nxt;
    }
    cur = nxt;
  }
  const cplx j0 = cmul(csin_dev(z), zinv);
  cplx jprev = cmul(rho[0], j0);
  cplx *o = reinterpret_cast<cplx *>(out);
  o[0] = jprev;
  o[1] = csub(j0, cmul(jprev, zinv));
  for (int i = 1; i < nmax; ++i) {
    const cplx ji = cmul(rho[i * rs], jprev);
    const cplx dji = csub(jprev, cmul(cscale(zinv, i + 1.), ji));
    cplx *oi = reinterpret_cast<cplx *>(out + i * stride);
    oi[0] = ji;
    oi[1] = dji;
    jprev = ji;
  }
}

// Node scalars follow GaussBasedResources::execute (GaussBasedResources.hpp:
// 132-152), get_r_dr_spheroid (SpecialFunctions.hpp:872-893) and
// InteractionTask::execute (InteractionResource.hpp:478-527).
// Tables of node g of one slot; kind 0: real-argument tables and node
// scalars, kind 1: complex-argument tables. Ratio columns in shared memory,
// i < rho_smem: the complex recurrence uses the complex entries tid + nt i
// of trho, the real one the doubles rtid + rnt i.
__device__ __forceinline__ void table_node(const TmxSlot &sl,
                                           const TmxGrain *__restrict__ grains,
                                           const double *__restrict__ gl_x,
                                           const double *__restrict__ gl_w,
                                           const int64_t *__restrict__ gl_off,
                                           double *tab, double *nsc,
                                           int bessel_start, int rho_smem,
                                           int g, int kind, cplx *trho, int tid,
                                           int nt, int rtid, int rnt) {
  const TmxGrain G = grains[sl.grain];
  const int N = sl.nmax;
  const int ng = sl.ngauss;
  const double *x = gl_x + gl_off[ng];
  const double *w = gl_w + gl_off[ng];
  {
    const double c = x[g];
    const double s2 = (1. - c) * (1. + c);
    const double sn = sqrt(s2);
    const double a2 = G.cbrt_d * G.cbrt_d;
    const double d2 = G.axis_ratio * G.axis_ratio;
    const double d2m1 = d2 - 1.;
    const double r2oa2 = 1. / (s2 + d2 * (c * c));
    const double r2 = a2 * r2oa2;
    const double drr = r2oa2 * c * sn * d2m1;
    const double r = sqrt(r2);
    double *T = tab + sl.tab + (int64_t)g * N * TMX_NQ;
    if (kind == 0) {
      const double kr = G.k * r * G.r_ev;
      const double krinv = 1. / kr;
      const cplx krmr = mkc(G.mr * G.k * r * G.r_ev, G.mi * G.k * r * G.r_ev);
      const cplx krmrinv = cinv(krmr);
      const double sin2inv = 1. / ((1. - c) * (1. + c));
      double *S = nsc + sl.nsc + (int64_t)g * TMX_NS;
      S[TMX_NS_KRINV] = krinv;
      S[TMX_NS_KRMRINV_RE] = krmrinv.x;
      S[TMX_NS_KRMRINV_IM] = krmrinv.y;
      S[TMX_NS_R2] = r2;
      S[TMX_NS_DRR] = drr;
      S[TMX_NS_W] = w[g];
      S[TMX_NS_COS] = c;
      S[TMX_NS_SININV] = sqrt(sin2inv);
      S[TMX_NS_SIN2INV] = sin2inv;
      S[TMX_NS_KR] = kr;
      S[TMX_NS_KRMR_RE] = krmr.x;
      S[TMX_NS_KRMR_IM] = krmr.y;
      // r^2 = d^{2/3} / (sin^2 + d^2 cos^2) (unit equal-volume radius):
      // d ln r^2 / dd = 2 / (3 d) - 2 d cos^2 / (sin^2 + d^2 cos^2);
      // r'/r = r2oa2 cos sin (d^2 - 1):
      // d(r'/r)/dd = 2 d cos sin r2oa2 (1 - cos^2 r2oa2 (d^2 - 1))
      const double dd = G.axis_ratio;
      S[TMX_NS_DLNR2_DD] = 2. / (3. * dd) - 2. * dd * (c * c) * r2oa2;
      S[TMX_NS_DDRR_DD] =
          2. * dd * c * sn * r2oa2 * (1. - (c * c) * r2oa2 * d2m1);
      S[TMX_NS_PAD] = 0.;
      S[TMX_NS_PAD2] = 0.;
      if (N <= rho_smem) {
        bessel_j_real(N, bessel_nstart(bessel_start, N, kr), kr, T + TMX_Q_J,
                      TMX_NQ, reinterpret_cast<double *>(trho) + rtid, rnt);
      } else {
        bessel_j_real(N, bessel_nstart(bessel_start, N, kr), kr, T + TMX_Q_J,
                      TMX_NQ, T + TMX_Q_J, TMX_NQ);
      }
      bessel_y_real(N, kr, T + TMX_Q_Y, TMX_NQ);
    } else {
      const cplx krmr = mkc(G.mr * G.k * r * G.r_ev, G.mi * G.k * r * G.r_ev);
      const int ns = bessel_nstart(bessel_start, N, hypot(krmr.x, krmr.y));
      if (N <= rho_smem) {
        bessel_j_complex(N, ns, krmr, T + TMX_Q_JM_RE, TMX_NQ, trho + tid, nt);
      } else {
        bessel_j_complex(N, ns, krmr, T + TMX_Q_JM_RE, TMX_NQ,
                         reinterpret_cast<cplx *>(T + TMX_Q_JM_RE), TMX_NQ / 2);
      }
    }
  }
}

// Grid (slot, node chunk, kind): kind 0 threads do the real-argument tables
// and node scalars of node g, kind 1 threads the complex-argument tables, so
// every warp runs one recurrence type.
__global__ void k_tables(const TmxSlot *__restrict__ slots, int nslots,
                         const TmxGrain *__restrict__ grains,
                         const double *__restrict__ gl_x,
                         const double *__restrict__ gl_w,
                         const int64_t *__restrict__ gl_off, double *tab,
                         double *nsc, int bessel_start, int rho_smem) {
  // ratio buffers: a shared-memory column per thread (rho_smem rows), or
  // the output slots themselves when the orders exceed rho_smem
  extern __shared__ cplx trho[];
  const int s = blockIdx.x;
  if (s >= nslots) {
    return;
  }
  const TmxSlot sl = slots[s];
  const int g = blockIdx.y * blockDim.x + threadIdx.x;
  if (g >= sl.ngauss) {
    return;
  }
  table_node(sl, grains, gl_x, gl_w, gl_off, tab, nsc, bessel_start, rho_smem, g,
             blockIdx.z, trho, threadIdx.x, blockDim.x, threadIdx.x, blockDim.x);
}

// Device-driven form (CUDA graph): the slots [0, *nact) of one order, whose
// count is known only on the device, as tasks of 32 nodes of one slot and
// one kind, one per warp at a time over a fixed grid; every slot of the
// launch has *ng_dev nodes. Same arithmetic per node as k_tables. The warps
// of a CTA may run different kinds, so a thread's real ratios stay inside
// its own complex column (every other double of it).
__global__ void k_tables_dev(const TmxSlot *__restrict__ slots, int nslots,
                             const int32_t *__restrict__ nact,
                             const int32_t *__restrict__ ng_dev,
                             const TmxGrain *__restrict__ grains,
                             const double *__restrict__ gl_x,
                             const double *__restrict__ gl_w,
                             const int64_t *__restrict__ gl_off, double *tab,
                             double *nsc, int bessel_start, int rho_smem) {
  extern __shared__ cplx trho[];
  const int ns = min(nslots, *nact);
  const int ng = *ng_dev;
  const int nch = (ng + 31) >> 5;
  const int64_t ntask = (int64_t)ns * nch * 2;
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int64_t t = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); t < ntask;
       t += (int64_t)gridDim.x * wpb) {
    const int s = (int)(t / (2 * nch));
    const int rem = (int)(t - (int64_t)s * 2 * nch);
    const int kind = rem & 1;
    const int g = (rem >> 1) * 32 + lane;
    const TmxSlot sl = slots[s];
    if (g < sl.ngauss) {
      table_node(sl, grains, gl_x, gl_w, gl_off, tab, nsc, bessel_start, rho_smem, g,
                 kind, trho, threadIdx.x, blockDim.x, 2 * threadIdx.x, 2 * blockDim.x);
    }
  }
}

// ---------------------------------------------------------------- Wigner --

// d^n_{0m}(x) and d/dx for n = 1..nmax by forward recurrence in n
// (SpecialFunctions::wigner_dn_0m, SpecialFunctions.hpp:302-371).
// out[(n-1) * 2 + {0,1}] = (d, dd)
__device__ static void wigner_d(double cosx, int nmax, int m, double *out) {
  const double sinx = sqrt((1. - cosx) * (1. + cosx));
  const double sinxinv = 1. / sinx;
  if (m == 0) {
    double d1 = 1.;
    double d2 = cosx;
    for (int n = 0; n < nmax; ++n) {
      const double np1 = n + 1.;
      const double np2 = n + 2.;
      const double np12p1 = 2. * np1 + 1.;
      const double dnp1 = (np12p1 * cosx * d2 - np1 * d1) / np2;
      const double ddn = sinxinv * np1 * np2 * (dnp1 - d1) / np12p1;
      out[2 * n] = d2;
      out[2 * n + 1] = ddn;
      d1 = d2;
      d2 = dnp1;
    }
    return;
  }
  const double m2 = (double)(m * m);
  double d1 = 0.;
  double d2 = 1.;
  for (int i = 0; i < m; ++i) {
    const double i2 = 2. * (i + 1.);
    d2 *= sqrt((i2 - 1.) / i2) * sinx;
  }
  for (int n = 0; n < m - 1; ++n) {
    out[2 * n] = 0.;
    out[2 * n + 1] = 0.;
  }
  for (int n = m - 1; n < nmax; ++n) {
    const double np1 = n + 1.;
    const double np2 = n + 2.;
    const double np12p1 = 2. * np1 + 1.;
    const double s12 = sqrt(np1 * np1 - m2);
    const double s22 = sqrt(np2 * np2 - m2);
    const double dnp1 = (np12p1 * cosx * d2 - s12 * d1) / s22;
    const double ddn = sinxinv * (np1 * s22 * dnp1 - np2 * s12 * d1) / np12p1;
    out[2 * n] = d2;
    out[2 * n + 1] = ddn;
    d1 = d2;
    d2 = dnp1;
  }
}

// Wigner tables at the lower-half quadrature nodes for one (nmax, ngauss):
// for orders below 100 the values are those of the mirrored upper-half node
// (cos = -x[g]) times (-1)^n (d) and -(-1)^n (dd), as WignerDResources
// precomputes them (WignerDResources.hpp:147-174); from order 100 on they are
// evaluated at the node itself (WignerDResources.hpp:232-247).
// out[((m - m_lo) * ng + g) * nmax * 2 + (n - 1) * 2 + {0,1}]
__global__ void k_wigner(const TmxWigJob *__restrict__ jobs, int njobs,
                         const double *__restrict__ gl_x,
                         const int64_t *__restrict__ gl_off, double *out) {
  const int j = blockIdx.y;
  if (j >= njobs) {
    return;
  }
  const TmxWigJob J = jobs[j];
  const int nm = J.m_hi - J.m_lo + 1;
  const int total = nm * J.ngauss;
  const double *x = gl_x + gl_off[J.ngauss];
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < total;
       u += gridDim.x * blockDim.x) {
    const int g = u % J.ngauss;
    const int m = J.m_lo + u / J.ngauss;
    double *o = out + J.out + ((int64_t)(m - J.m_lo) * J.ngauss + g) *
                                  J.nmax * 2;
    if (J.nmax < 100) {
      wigner_d(-x[g], J.nmax, m, o);
      double sign = 1.;
      for (int n = 0; n < J.nmax; ++n) {
        sign = -sign;
        o[2 * n] = sign * o[2 * n];
        o[2 * n + 1] = -sign * o[2 * n + 1];
      }
    } else {
      wigner_d(x[g], J.nmax, m, o);
    }
  }
}

// --------------------------------------------------------- launchers ------

void tmx_launch_tables(const TmxSlot *slots, int nslots, const TmxGrain *grains,
                       const double *gl_x, const double *gl_w,
                       const int64_t *gl_off, double *tab, double *nsc,
                       int bessel_start, int ngmax, int nmax_max,
                       cudaStream_t stream) {
  if (nslots <= 0 || ngmax <= 0) {
    return;
  }
  // one thread per node: a warp per slot and argument kind when every slot
  // has at most 32 nodes (the order loop up to order 16), else chunks of 64
  const int threads = (ngmax <= 32) ? 32 : 64;
  // ratios in shared memory for orders up to 48, sized by the launch's
  // largest order (more CTAs per SM for small orders)
  const int rho_smem = std::max(1, std::min(48, nmax_max));
  const size_t smem = (size_t)threads * rho_smem * sizeof(cplx);
  static int attr_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaFuncSetAttribute(k_tables, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(64 * 48 * sizeof(cplx)));
    attr_dev = dev;
  }
  dim3 grid(nslots, (ngmax + threads - 1) / threads, 2);
  k_tables<<<grid, threads, smem, stream>>>(slots, nslots, grains, gl_x, gl_w,
                                            gl_off, tab, nsc, bessel_start,
                                            rho_smem);
}

void tmx_launch_tables_dev(const TmxSlot *slots, int nslots, const int32_t *nact,
                           const int32_t *ng_dev, const TmxGrain *grains,
                           const double *gl_x, const double *gl_w,
                           const int64_t *gl_off, double *tab, double *nsc,
                           int bessel_start, int nmax_max, cudaStream_t stream) {
  if (nslots <= 0) {
    return;
  }
  // two warps per CTA; ratios in shared memory for orders up to 48
  const int threads = 64;
  const int rho_smem = std::max(1, std::min(48, nmax_max));
  const size_t smem = (size_t)threads * rho_smem * sizeof(cplx);
  static int attr_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaFuncSetAttribute(k_tables_dev, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(64 * 48 * sizeof(cplx)));
    attr_dev = dev;
  }
  // resident CTAs only (shared memory allows four per SM at orders >= 48)
  const int blocks = 148 * 4;
  k_tables_dev<<<blocks, threads, smem, stream>>>(slots, nslots, nact, ng_dev, grains,
                                                  gl_x, gl_w, gl_off, tab, nsc,
                                                  bessel_start, rho_smem);
}

void tmx_launch_wigner(const TmxWigJob *jobs, int njobs, int max_work,
                       const double *gl_x, const int64_t *gl_off, double *out,
                       cudaStream_t stream) {
  if (njobs <= 0) {
    return;
  }
  const int threads = 128;
  int bx = (max_work + threads - 1) / threads;
  if (bx < 1) {
    bx = 1;
  }
  dim3 grid(bx, njobs);
  k_wigner<<<grid, threads, 0, stream>>>(jobs, njobs, gl_x, gl_off, out);
}
