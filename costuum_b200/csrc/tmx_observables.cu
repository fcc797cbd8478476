// Observables of (orientation-averaged) T-matrices on device (sm_100a, FP64).
//
//   k_cg            Clebsch-Gordan rows <n1 m n2 -m | N 0>, m >= 0
//                   (SpecialFunctions::get_clebsch_gordan_coefficients,
//                   SpecialFunctions.hpp:1131-1244)
//   k_orient_avg    AlignmentAverageTask::execute (AlignmentAverageTask.hpp:
//                   115-215), restructured: the m1 sum does not depend on m,
//                   so it is formed once per (n1, n2, N) and reused for every
//                   m (O(N^4) instead of O(N^5))
//   k_forward_s     the forward-scattering amplitude S of
//                   ExtinctionCoefficientTask.hpp:517-619 (and its copies in
//                   AbsorptionCoefficientTask.hpp:612-715 and
//                   ScatteringMatrixTask.hpp:588-691) for one (theta_in,
//                   theta_out) pair and a list of azimuths: the per-m sums
//                   over (n, n') are formed once, each azimuth then costs
//                   O(nmax)
//   k_q_epilogue    Q_ext/Q_extpol/Q_extcpol and Q_abs/Q_abspol (with the
//                   optional scattering subtraction of
//                   AbsorptionCoefficientTask.hpp:742-773)
//   k_z_epilogue    4x4 scattering matrix (ScatteringMatrixTask.hpp:719-748)
//   k_shape_avg     ShapeAveragingTask (ShapeAveragingTask.hpp:127-166)
//
// Compiled with --fmad=false, like the table kernels, so the recurrences
// round as the reference's build does.
#include <algorithm>

#include "tmx_common.cuh"
#include "tmx_kernels.h"

// ---------------------------------------------------------- CG table -----

// offset table: cg_off[(n1 - 1) * nmax + (n2 - 1)] -> start of the pair's
// rows; row N (|n1-n2| <= N <= n1+n2) holds min(n1,n2) + 1 values, m = 0..min
__device__ static void cg_row(int nmax, int pair, int Ni,
                              const int64_t *__restrict__ cg_off,
                              double *__restrict__ cg, double *rowA,
                              double *rowB) {
  const int n1 = pair / nmax + 1;
  const int n2 = pair % nmax + 1;
  const int M = min(n1, n2);
  const int Nlo = abs(n1 - n2);
  const int N = Nlo + Ni;
  if (N > n1 + n2) {
    return;
  }
  const int nsize = 2 * n1 + 1;
  for (int i = 0; i < nsize; ++i) {
    rowA[i] = 0.;
    rowB[i] = 0.;
  }
  // upper row M = N
  double *top = rowA;
  top[n1 + n1] = 1.;
  double norm = 1.;
  const int lo = max(-n1, N - n2 - 1);
  for (int m1t = n1 - 1; m1t >= lo; --m1t) {
    const double cp2 = sqrt((n2 - N + m1t + 1.) * (n2 + N - m1t));
    const double cp1 = sqrt((n1 - m1t) * (n1 + m1t + 1.));
    const double cnext = -cp2 * top[m1t + 1 + n1] / cp1;
    top[m1t + n1] = cnext;
    norm += cnext * cnext;
  }
  const double inv_norm = 1. / sqrt(norm);
  for (int m1t = n1; m1t >= lo; --m1t) {
    top[m1t + n1] *= inv_norm;
  }
  double *prev = rowA, *cur = rowB;
  for (int Mt = N - 1; Mt >= 0; --Mt) {
    const double cmin_inv = 1. / sqrt((N + Mt + 1.) * (N - Mt));
    const int a = max(-n1, Mt - n2);
    const int b = min(n1, Mt + n2);
    for (int m1t = a; m1t <= b; ++m1t) {
      const int m2t = Mt - m1t;
      double t1 = 0.;
      if (m1t + 1 <= n1) {
        t1 = sqrt((n1 + m1t + 1.) * (n1 - m1t)) * prev[m1t + 1 + n1];
      }
      double t2 = 0.;
      if (m2t + 1 <= n2) {
        t2 = sqrt((n2 + m2t + 1.) * (n2 - m2t)) * prev[m1t + n1];
      }
      cur[m1t + n1] = cmin_inv * (t1 + t2);
    }
    double *t = prev;
    prev = cur;
    cur = t;
  }
  // prev holds row M = 0; keep m = 0..M
  double *o = cg + cg_off[pair] + (int64_t)(N - Nlo) * (M + 1);
  for (int m = 0; m <= M; ++m) {
    o[m] = prev[m + n1];
  }
}

__global__ void k_cg(int nmax, const int64_t *__restrict__ cg_off,
                     double *__restrict__ cg, double *__restrict__ work) {
  const int npairs = nmax * nmax;
  const int rows = 2 * nmax + 1; // at most 2 nmax + 1 values of N per pair
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  const int wlen = 2 * nmax + 1;
  // two rolling rows of the ladder recursion in this thread's work slot
  double *rowA = work + (int64_t)slot * 2 * wlen;
  double *rowB = rowA + wlen;
  for (int64_t u = slot; u < (int64_t)npairs * rows;
       u += (int64_t)gridDim.x * blockDim.x) {
    cg_row(nmax, (int)(u / rows), (int)(u % rows), cg_off, cg, rowA, rowB);
  }
}

// ------------------------------------------------- orientation average ---

__device__ __forceinline__ int64_t tblock(int N, int m) {
  if (m == 0) {
    return 0;
  }
  const int64_t a = N, b = N + 1 - m;
  return 4 * (a * a + a * (a + 1) * (2 * a + 1) / 6 - b * (b + 1) * (2 * b + 1) / 6);
}

// element (i1, n1; i2, n2) of block m of a T-matrix of order N
__device__ __forceinline__ int64_t telem(int N, int m, int i1, int n1, int i2,
                                         int n2) {
  const int nb = (m == 0) ? N : N + 1 - m;
  const int nmin = (m == 0) ? 1 : m;
  return tblock(N, m) + (int64_t)(i1 * nb + n1 - nmin) * (2 * nb) + i2 * nb +
         n2 - nmin;
}

// acc += t * a (complex times real), fused; this file is compiled without
// automatic contraction, so the contractions are spelled out
__device__ __forceinline__ void cfma(cplx &acc, cplx t, double a) {
  acc.x = __fma_rn(t.x, a, acc.x);
  acc.y = __fma_rn(t.y, a, acc.y);
}

// sqrt((2n + 1) / ((n + 1) n)), the factor of a_{n n'} for one order
__device__ __forceinline__ double a_fac(int n) {
  return sqrt((2. * n + 1.) / ((n + 1.) * n));
}

// c_{n' n} z for c_{n' n} = i^{n' - n - 1} a_{n' n} (NBasedResources::get_cnn,
// NBasedResources.hpp:115-137); n' is the incoming order (column), n the
// outgoing one (row)
__device__ __forceinline__ cplx c_fold(int nin, int nout, double a, cplx z) {
  const cplx s = cscale(z, a);
  switch ((((nin - nout - 1) % 4) + 4) % 4) {
  case 0:
    return s;
  case 1:
    return mkc(-s.y, s.x);
  case 2:
    return mkc(-s.x, -s.y);
  default:
    return mkc(s.y, -s.x);
  }
}

// One warp per (grain, n1, n2). AlignmentAverageTask::execute (Alignment
// AverageTask.hpp:115-215) forms, for every m,
//   Ta_m = sum_N' p_N' (-1)^m CG(n1 m n2 -m|N'0) sum_m1 f(m1) (-1)^m1
//          CG(n1 m1 n2 -m1|N'0) T_m1,
// with f = 1 for m1 = 0 and 2 otherwise; the m1 sum does not depend on m, so
// pass 1 forms it once per N' (lanes over N') and pass 2 contracts over N'
// (lanes over m): O(n^2) per pair instead of O(n^3). Even N' - |n1 - n2|
// couple the (0,0) and (1,1) sub-blocks, odd ones (0,1) and (1,0). Grains
// without an orientation distribution (coef_set < 0) are copied. Either way
// the output carries the factor c_{n2 n1} of the amplitude sums, so that
// the amplitude kernel contracts Ta with real vectors only.
// Shared memory per warp and matrix: t[4][M + 1] and S[2][2M + 1] complex.
// NMAT matrices (a T-matrix and its tangents) share the Clebsch-Gordan
// reads and the loops; each is summed in the same order as alone.
template <int NMAT>
__global__ void __launch_bounds__(256)
k_orient_pairs(const TmxObsGrain *__restrict__ og,
               const int64_t *__restrict__ pstart,
               const int32_t *__restrict__ order, int pmax,
               int64_t npairs, TmxMatSet mats, const double *__restrict__ coeffs,
               int ncoef, const int64_t *__restrict__ cg_off,
               const double *__restrict__ cg, int cg_nmax, int wcap, int fold) {
  extern __shared__ cplx osh[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  cplx *tv = osh + (int64_t)warp * wcap * NMAT;
  for (int64_t w = (int64_t)blockIdx.x * nwarps + warp; w < npairs;
       w += (int64_t)gridDim.x * nwarps) {
    // work item w = (pair (n1, n2), grain): pair-major, so that the warps
    // of a CTA (and CTAs running together) contract the same Clebsch-Gordan
    // rows for different grains and read them from cache. Pair
    // q = (n1 - 1) pmax + (n2 - 1) owns items [pstart[q], pstart[q + 1]),
    // one per grain of order >= max(n1, n2), in the order `order` (grains by
    // descending order).
    int lo = 0, hi = pmax * pmax - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pstart[mid] <= w) {
        lo = mid;
      } else {
        hi = mid - 1;
      }
    }
    const int n1 = lo / pmax + 1;
    const int n2 = lo % pmax + 1;
    const TmxObsGrain G = og[order[w - pstart[lo]]];
    const int N = G.nmax;
    const int M = min(n1, n2);
    // fold = 0: the plain averaged T-matrix (c = 1: i^0 times 1)
    const double afold = fold ? a_fac(n1) * a_fac(n2) : 1.;
    const int nfold = fold ? n1 : n2 - 1;
    if (G.coef_set < 0) {
      for (int m = lane; m <= M; m += 32) {
        for (int q = 0; q < 4; ++q) {
          const int i1 = q >> 1, i2 = q & 1;
          const int64_t e = telem(N, m, i1, n1, i2, n2);
#pragma unroll
          for (int k = 0; k < NMAT; ++k) {
            mats.dst[k][G.t_off + e] = c_fold(n2, nfold, afold, mats.src[k][G.t_off + e]);
          }
        }
      }
      continue;
    }
    const double *p = coeffs + (int64_t)G.coef_set * ncoef;
    const int nN = 2 * M + 1;
    const int Nlo = abs(n1 - n2);
    const double *C = cg + cg_off[(n1 - 1) * cg_nmax + (n2 - 1)];
    // per matrix k: t00, t11, t01, t10 [M + 1] and S [2 (2M + 1)] at tv + k wcap
    const int o11 = M + 1, o01 = 2 * (M + 1), o10 = 3 * (M + 1), oS = 4 * (M + 1);
    for (int m1 = lane; m1 <= M; m1 += 32) {
      // f(m1) (-1)^m1 is a power of two with a sign: the product is exact
      const double f = ((m1 == 0) ? 1. : 2.) * ((m1 & 1) ? -1. : 1.);
#pragma unroll
      for (int k = 0; k < NMAT; ++k) {
        const cplx *Tg = mats.src[k] + G.t_off;
        cplx *t = tv + k * wcap;
        t[m1] = cscale(Tg[telem(N, m1, 0, n1, 0, n2)], f);
        t[o11 + m1] = cscale(Tg[telem(N, m1, 1, n1, 1, n2)], f);
        t[o01 + m1] = cscale(Tg[telem(N, m1, 0, n1, 1, n2)], f);
        t[o10 + m1] = cscale(Tg[telem(N, m1, 1, n1, 0, n2)], f);
      }
    }
    __syncwarp();
    // pass 1: S(N') for the two sub-blocks of its parity
    for (int j = lane; j < nN; j += 32) {
      const double *Cr = C + (int64_t)j * (M + 1);
      const int oa = (j & 1) ? o01 : 0;
      const int ob = (j & 1) ? o10 : o11;
      cplx sa[NMAT], sb[NMAT];
#pragma unroll
      for (int k = 0; k < NMAT; ++k) {
        sa[k] = sb[k] = mkc(0., 0.);
      }
      for (int m1 = 0; m1 <= M; ++m1) {
        const double c = Cr[m1];
#pragma unroll
        for (int k = 0; k < NMAT; ++k) {
          cfma(sa[k], tv[k * wcap + oa + m1], c);
          cfma(sb[k], tv[k * wcap + ob + m1], c);
        }
      }
#pragma unroll
      for (int k = 0; k < NMAT; ++k) {
        tv[k * wcap + oS + 2 * j] = sa[k];
        tv[k * wcap + oS + 2 * j + 1] = sb[k];
      }
    }
    __syncwarp();
    // pass 2: Ta_m = sum_N' p_N' (-1)^m CG(m) S(N')
    for (int m = lane; m <= M; m += 32) {
      cplx e00[NMAT], e11[NMAT], e01[NMAT], e10[NMAT];
#pragma unroll
      for (int k = 0; k < NMAT; ++k) {
        e00[k] = e11[k] = e01[k] = e10[k] = mkc(0., 0.);
      }
      const double ms = (m & 1) ? -1. : 1.;
      for (int j = 0; j < nN; j += 2) {
        const double f = ms * p[Nlo + j] * C[(int64_t)j * (M + 1) + m];
#pragma unroll
        for (int k = 0; k < NMAT; ++k) {
          cfma(e00[k], tv[k * wcap + oS + 2 * j], f);
          cfma(e11[k], tv[k * wcap + oS + 2 * j + 1], f);
        }
      }
      for (int j = 1; j < nN; j += 2) {
        const double f = ms * p[Nlo + j] * C[(int64_t)j * (M + 1) + m];
#pragma unroll
        for (int k = 0; k < NMAT; ++k) {
          cfma(e01[k], tv[k * wcap + oS + 2 * j], f);
          cfma(e10[k], tv[k * wcap + oS + 2 * j + 1], f);
        }
      }
#pragma unroll
      for (int k = 0; k < NMAT; ++k) {
        cplx *Tag = mats.dst[k] + G.t_off;
        Tag[telem(N, m, 0, n1, 0, n2)] = c_fold(n2, nfold, afold, e00[k]);
        Tag[telem(N, m, 1, n1, 1, n2)] = c_fold(n2, nfold, afold, e11[k]);
        Tag[telem(N, m, 0, n1, 1, n2)] = c_fold(n2, nfold, afold, e01[k]);
        Tag[telem(N, m, 1, n1, 0, n2)] = c_fold(n2, nfold, afold, e10[k]);
      }
    }
    __syncwarp();
  }
}

// -------------------------------------------------- forward amplitude ----

// pi_n = m d^n_{0m}(x) / sin x and tau_n = d/dx d^n_{0m}(x) for one m and
// n = nmin..nmax, written to pi[(n - nmin) * stride], tau[...]
// (SpecialFunctions::wigner_dn_0m_sinx, SpecialFunctions.hpp:397-495)
__device__ static void wigner_col(double cosx, double sinx, double sinx_inv,
                                  int nmax, int m, double *pi, double *tau,
                                  int stride) {
  const int nmin = (m > 1) ? m : 1;
  if (fabs(1. - fabs(cosx)) <= 1.e-10) {
    if (m == 1) {
      int sign = 1;
      for (int n = 1; n < nmax + 1; ++n) {
        double dn = 0.5 * sqrt(n * (n + 1.));
        if (cosx < 0.) {
          dn *= sign;
        }
        pi[(n - nmin) * stride] = m * dn;
        if (cosx < 0.) {
          dn = -dn;
        }
        tau[(n - nmin) * stride] = dn;
        sign = -sign;
      }
    } else {
      for (int n = nmin; n <= nmax; ++n) {
        pi[(n - nmin) * stride] = 0.;
        tau[(n - nmin) * stride] = 0.;
      }
    }
    return;
  }
  if (m == 0) {
    double d1 = 1.;
    double d2 = cosx;
    for (int n = 0; n < nmax; ++n) {
      const double np1 = n + 1.;
      const double np2 = n + 2.;
      const double np12p1 = 2. * np1 + 1.;
      const double dnp1 = (np12p1 * cosx * d2 - np1 * d1) / np2;
      const double ddn = sinx_inv * np1 * np2 * (dnp1 - d1) / np12p1;
      pi[n * stride] = 0.;
      tau[n * stride] = ddn;
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
  for (int n = m - 1; n < nmax; ++n) {
    const double np1 = n + 1.;
    const double np2 = n + 2.;
    const double np12p1 = 2. * np1 + 1.;
    const double s12 = sqrt(np1 * np1 - m2);
    const double s22 = sqrt(np2 * np2 - m2);
    const double dnp1 = (np12p1 * cosx * d2 - s12 * d1) / s22;
    const double ddn = sinx_inv * (np1 * s22 * dnp1 - np2 * s12 * d1) / np12p1;
    pi[(n + 1 - nmin) * stride] = m * (d2 * sinx_inv);
    tau[(n + 1 - nmin) * stride] = ddn;
    d1 = d2;
    d2 = dnp1;
  }
}

// pi and tau columns of every (angle, m <= nmax) of an amplitude plan, the
// recurrence of k_amp done once for all grains and jobs that share an angle:
// column (a, m) holds orders n = max(m, 1) .. nmax at ((a (nmax + 1) + m)
// nmax). (The values of orders <= N do not depend on how far the
// recurrence runs, so a grain of order N reads the first entries.)
__global__ void k_wigner_cols(const TmxAngle *__restrict__ angles, int nangles,
                              int nmax, double *pi, double *tau) {
  const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= (int64_t)nangles * (nmax + 1)) {
    return;
  }
  const int a = (int)(u / (nmax + 1));
  const int m = (int)(u - (int64_t)a * (nmax + 1));
  const TmxAngle A = angles[a];
  wigner_col(A.c, A.s, A.si, nmax, m, pi + u * nmax, tau + u * nmax, 1);
}

// One CTA per group of up to 32 amplitude jobs of one grain (lane = job).
// For every m, with u = (pi_n, tau_n) at the outgoing angle and v at the
// incoming one (n the row order, n' the column order of block m),
//   X0 = u^T Tc v,  X1 = u^T Tc v',  X2 = u'^T Tc v,  X3 = u'^T Tc v'
// where Tc is block m with the c_{n' n} factors folded in and u', v' swap
// the pi and tau halves: the four (n, n') sums of
// ExtinctionCoefficientTask.hpp:517-619 as one (2nb x 2nb) x (2nb x 64)
// product per m. Warps own rows; lanes own jobs; the T row is read once per
// warp (a broadcast) and the angle vectors come from shared memory. X is
// kept in this CTA's global slot; the azimuth pass then forms
//   S = (1/k) sum_m (2 cos m phi, 2 sin m phi) X_m
// with e^{i m phi} built by repeated multiplication as in the reference.
template <int NMAT>
__global__ void __launch_bounds__(256, (NMAT > 1) ? 2 : 3)
k_amp(const TmxAmpGroup *__restrict__ groups, int ngroups,
      const TmxSJob *__restrict__ jobs, const TmxObsGrain *__restrict__ og,
      TmxMatSet mats, const TmxAngle *__restrict__ angles,
      const cplx *__restrict__ phis, cplx *__restrict__ xslot, int nbmax,
      const double *__restrict__ wpi, const double *__restrict__ wtau,
      int wnmax) {
  extern __shared__ double ash[];
  double *po = ash;
  double *to = po + nbmax * 32;
  double *pi = to + nbmax * 32;
  double *ti = pi + nbmax * 32;
  cplx *red = (cplx *)(ti + nbmax * 32); // [NMAT][8 warps][4][32 lanes]
  __shared__ TmxSJob sj[32];
  __shared__ int pref[33];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  cplx *X = xslot + (int64_t)blockIdx.x * 32 * (nbmax + 1) * 4 * NMAT;
  for (int gi = blockIdx.x; gi < ngroups; gi += gridDim.x) {
    const TmxAmpGroup grp = groups[gi];
    const TmxObsGrain G = og[grp.grain];
    const int N = G.nmax;
    const int nj = grp.njobs;
    if (tid < nj) {
      sj[tid] = jobs[grp.job0 + tid];
    }
    __syncthreads();
    if (tid == 0) {
      pref[0] = 0;
      for (int p = 0; p < nj; ++p) {
        pref[p + 1] = pref[p] + sj[p].nphi;
      }
    }
    for (int m = 0; m <= N; ++m) {
      const int nmin = (m > 1) ? m : 1;
      const int nb = N + 1 - nmin;
      if (wpi) {
        // the columns of this m from the plan's table (k_wigner_cols)
        for (int u = tid; u < 64 * nb; u += blockDim.x) {
          const int side = u / (32 * nb); // 0: outgoing angle, 1: incoming
          const int k = (u - side * 32 * nb) >> 5;
          const int p = u & 31;
          double pv = 0., tv = 0.;
          if (p < nj) {
            const int a = side ? sj[p].angle_in : sj[p].angle_out;
            const int64_t off = ((int64_t)a * (wnmax + 1) + m) * wnmax + k;
            pv = wpi[off];
            tv = wtau[off];
          }
          (side ? pi : po)[k * 32 + p] = pv;
          (side ? ti : to)[k * 32 + p] = tv;
        }
      } else if (tid < 64) {
        const int p = tid & 31;
        const int side = tid >> 5; // 0: outgoing angle, 1: incoming angle
        double *P = side ? pi : po;
        double *Tt = side ? ti : to;
        if (p < nj) {
          const TmxAngle a = angles[side ? sj[p].angle_in : sj[p].angle_out];
          wigner_col(a.c, a.s, a.si, N, m, P + p, Tt + p, 32);
        } else {
          for (int k = 0; k < nb; ++k) {
            P[k * 32 + p] = 0.;
            Tt[k * 32 + p] = 0.;
          }
        }
      }
      __syncthreads();
      cplx x0[NMAT], x1[NMAT], x2[NMAT], x3[NMAT];
#pragma unroll
      for (int q = 0; q < NMAT; ++q) {
        x0[q] = x1[q] = x2[q] = x3[q] = mkc(0., 0.);
      }
      const int64_t tb = G.t_off + tblock(N, m);
      for (int r = warp; r < 2 * nb; r += 8) {
        cplx y0[NMAT], y1[NMAT];
#pragma unroll
        for (int q = 0; q < NMAT; ++q) {
          y0[q] = y1[q] = mkc(0., 0.);
        }
#pragma unroll 4
        for (int k = 0; k < nb; ++k) {
          const double a = pi[k * 32 + lane];
          const double b = ti[k * 32 + lane];
#pragma unroll
          for (int q = 0; q < NMAT; ++q) {
            const cplx *Tr = mats.src[q] + tb + (int64_t)r * 2 * nb;
            const cplx t0 = Tr[k];
            const cplx t1 = Tr[nb + k];
            cfma(y0[q], t0, a);
            cfma(y0[q], t1, b);
            cfma(y1[q], t0, b);
            cfma(y1[q], t1, a);
          }
        }
        const int kr = (r < nb) ? r : r - nb;
        const double u = (r < nb) ? po[kr * 32 + lane] : to[kr * 32 + lane];
        const double up = (r < nb) ? to[kr * 32 + lane] : po[kr * 32 + lane];
#pragma unroll
        for (int q = 0; q < NMAT; ++q) {
          cfma(x0[q], y0[q], u);
          cfma(x1[q], y1[q], u);
          cfma(x2[q], y0[q], up);
          cfma(x3[q], y1[q], up);
        }
      }
#pragma unroll
      for (int q = 0; q < NMAT; ++q) {
        cplx *rq = red + q * 8 * 4 * 32;
        rq[(warp * 4 + 0) * 32 + lane] = x0[q];
        rq[(warp * 4 + 1) * 32 + lane] = x1[q];
        rq[(warp * 4 + 2) * 32 + lane] = x2[q];
        rq[(warp * 4 + 3) * 32 + lane] = x3[q];
      }
      __syncthreads();
      for (int v = tid; v < 128 * NMAT; v += blockDim.x) {
        const int q = v >> 7;
        const int k = (v >> 5) & 3;
        const cplx *rq = red + q * 8 * 4 * 32;
        cplx s = rq[k * 32 + lane];
        for (int w = 1; w < 8; ++w) {
          s = cadd(s, rq[(w * 4 + k) * 32 + lane]);
        }
        if (lane < nj) {
          X[(((int64_t)q * 32 + lane) * (N + 1) + m) * 4 + k] = s;
        }
      }
    }
    __syncthreads();
    const double kinv = 1. / G.k;
    for (int item = tid; item < pref[nj]; item += blockDim.x) {
      int p = 0;
      while (pref[p + 1] <= item) {
        ++p;
      }
      const TmxSJob J = sj[p];
      const int f = item - pref[p];
      const cplx e1 = phis[J.phi0 + f];
#pragma unroll
      for (int q = 0; q < NMAT; ++q) {
        const cplx *Xp = X + ((int64_t)q * 32 + p) * (N + 1) * 4;
        cplx e = mkc(1., 0.);
        cplx s0 = mkc(0., 0.), s1 = s0, s2 = s0, s3 = s0;
        for (int m = 0; m <= N; ++m) {
          const double fcos = 2. * e.x;
          const double fsin = 2. * e.y;
          e = cmul(e, e1);
          if (m == 0) {
            s0 = cadd(s0, Xp[0]);
            s3 = cadd(s3, Xp[3]);
          } else {
            s0 = cadd(s0, cscale(Xp[m * 4 + 0], fcos));
            s1 = cadd(s1, cscale(Xp[m * 4 + 1], fsin));
            s2 = csub(s2, cscale(Xp[m * 4 + 2], fsin));
            s3 = cadd(s3, cscale(Xp[m * 4 + 3], fcos));
          }
        }
        cplx *o = mats.dst[q] + (J.out + f) * 4;
        o[0] = cscale(s0, kinv);
        o[1] = cscale(s1, kinv);
        o[2] = cscale(s2, kinv);
        o[3] = cscale(s3, kinv);
      }
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------- epilogues ---

__device__ __forceinline__ double zsum(const cplx *S, double s1, double s2,
                                       double s3) {
  // 0.5 (|S0|^2 + s1 |S1|^2 + s2 |S2|^2 + s3 |S3|^2)
  return 0.5 * (cnorm2(S[0]) + s1 * cnorm2(S[1]) + s2 * cnorm2(S[2]) +
                s3 * cnorm2(S[3]));
}

// One thread per (grain, theta): extinction and absorption coefficients from
// the theta -> theta amplitude, minus the directional scattering integral
// when requested (the reference subtracts sum_{theta', phi'} w Z00 and Z10).
__global__ void k_q_epilogue(const TmxQJob *__restrict__ jobs, int njobs,
                             const TmxObsGrain *__restrict__ og,
                             const cplx *__restrict__ S,
                             const double *__restrict__ wts, int nacc,
                             double *__restrict__ qout, int qstride,
                             int do_abs, int do_ext) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= njobs) {
    return;
  }
  const TmxQJob J = jobs[u];
  const TmxObsGrain G = og[J.grain];
  const cplx *s = S + J.s_main * 4;
  const double prefactor = 2. * M_PI / G.k;
  const double norm = M_PI * G.r_ev * G.r_ev;
  double *o = qout + (int64_t)J.out * qstride;
  int k = 0;
  if (do_abs) {
    double qabs = prefactor * (s[0].y + s[3].y);
    double qabspol = prefactor * (s[0].y - s[3].y);
    if (nacc > 0) {
      for (int t = 0; t < nacc; ++t) {
        for (int p = 0; p < nacc; ++p) {
          const cplx *st = S + (J.s_acc + (int64_t)t * nacc + p) * 4;
          const double w = wts[t] * wts[nacc + p];
          qabs -= zsum(st, 1., 1., 1.) * w;
          qabspol -= zsum(st, 1., -1., -1.) * w;
        }
      }
    }
    o[k++] = qabs / norm;
    o[k++] = qabspol / norm;
  }
  if (do_ext) {
    o[k++] = prefactor * (s[0].y + s[3].y) / norm;
    o[k++] = prefactor * (s[0].y - s[3].y) / norm;
    o[k++] = prefactor * (s[3].x - s[0].x) / norm;
  }
}

// One thread per (grain, theta): derivatives of (Qext, Qextpol, Qextcpol)
// with respect to (Re m, Im m, R_V, d) from the tangent amplitudes. S is
// linear in T, and T is holomorphic in m, so dS/d(Im m) = i dS/d(Re m); the
// normalisation 1/(pi R_V^2) adds -2 Q / R_V to the R_V derivative.
// dq[(job.out * 3 + k) * 4 + p]
__global__ void k_dq_epilogue(const TmxQJob *__restrict__ jobs, int njobs,
                              const TmxObsGrain *__restrict__ og,
                              const cplx *__restrict__ S,
                              const cplx *__restrict__ dSm,
                              const cplx *__restrict__ dSr,
                              const cplx *__restrict__ dSd,
                              double *__restrict__ dq) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= njobs) {
    return;
  }
  const TmxQJob J = jobs[u];
  const TmxObsGrain G = og[J.grain];
  const double f = (2. * M_PI / G.k) / (M_PI * G.r_ev * G.r_ev);
  const cplx *s = S + J.s_main * 4;
  const double q[3] = {f * (s[0].y + s[3].y), f * (s[0].y - s[3].y),
                       f * (s[3].x - s[0].x)};
  const cplx *dm = dSm + J.s_main * 4;
  const cplx *dr = dSr + J.s_main * 4;
  const cplx *dd = dSd + J.s_main * 4;
  double *o = dq + J.out * 12;
  // Re m
  o[0 * 4 + 0] = f * (dm[0].y + dm[3].y);
  o[1 * 4 + 0] = f * (dm[0].y - dm[3].y);
  o[2 * 4 + 0] = f * (dm[3].x - dm[0].x);
  // Im m: Im(i z) = Re z, Re(i z) = -Im z
  o[0 * 4 + 1] = f * (dm[0].x + dm[3].x);
  o[1 * 4 + 1] = f * (dm[0].x - dm[3].x);
  o[2 * 4 + 1] = -f * (dm[3].y - dm[0].y);
  // R_V
  o[0 * 4 + 2] = f * (dr[0].y + dr[3].y) - 2. * q[0] / G.r_ev;
  o[1 * 4 + 2] = f * (dr[0].y - dr[3].y) - 2. * q[1] / G.r_ev;
  o[2 * 4 + 2] = f * (dr[3].x - dr[0].x) - 2. * q[2] / G.r_ev;
  // axis ratio
  o[0 * 4 + 3] = f * (dd[0].y + dd[3].y);
  o[1 * 4 + 3] = f * (dd[0].y - dd[3].y);
  o[2 * 4 + 3] = f * (dd[3].x - dd[0].x);
}

// one thread per (grain, theta_out, phi_out): the 4x4 matrix of
// ScatteringMatrixTask::execute from S, row major
__global__ void k_z_epilogue(int n, const cplx *__restrict__ S,
                             double *__restrict__ zout) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) {
    return;
  }
  const cplx *s = S + (int64_t)u * 4;
  const cplx S0 = s[0], S1 = s[1], S2 = s[2], S3 = s[3];
  auto cj = [](cplx a) { return mkc(a.x, -a.y); };
  auto re_i = [](cplx a) { return -a.y; }; // Re(i a)
  double *Z = zout + (int64_t)u * 16;
  Z[0] = zsum(s, 1., 1., 1.);
  Z[1] = 0.5 * (cnorm2(S0) - cnorm2(S1) + cnorm2(S2) - cnorm2(S3));
  Z[2] = (csub(mkc(0., 0.), cadd(cmul(S0, cj(S1)), cmul(S3, cj(S2))))).x;
  Z[3] = re_i(csub(cmul(S0, cj(S1)), cmul(S3, cj(S2))));
  Z[4] = 0.5 * (cnorm2(S0) + cnorm2(S1) - cnorm2(S2) - cnorm2(S3));
  Z[5] = 0.5 * (cnorm2(S0) - cnorm2(S1) - cnorm2(S2) + cnorm2(S3));
  Z[6] = (cadd(mkc(-cmul(S0, cj(S1)).x, -cmul(S0, cj(S1)).y),
               cmul(S3, cj(S2)))).x;
  Z[7] = re_i(cadd(cmul(S0, cj(S1)), cmul(S3, cj(S2))));
  Z[8] = (csub(mkc(-cmul(S0, cj(S2)).x, -cmul(S0, cj(S2)).y),
               cmul(S3, cj(S1)))).x;
  Z[9] = (cadd(mkc(-cmul(S0, cj(S2)).x, -cmul(S0, cj(S2)).y),
               cmul(S3, cj(S1)))).x;
  Z[10] = cadd(cmul(S0, cj(S3)), cmul(S1, cj(S2))).x;
  Z[11] = -re_i(cadd(cmul(S0, cj(S3)), cmul(S2, cj(S1))));
  Z[12] = re_i(cadd(cmul(S2, cj(S0)), cmul(S3, cj(S1))));
  Z[13] = re_i(csub(cmul(S2, cj(S0)), cmul(S3, cj(S1))));
  Z[14] = -re_i(csub(cmul(S3, cj(S0)), cmul(S1, cj(S2))));
  Z[15] = csub(cmul(S3, cj(S0)), cmul(S1, cj(S2))).x;
}

// shape average: out[c][j] = sum_s w_s in[c][s][j] / sum_s w_s
__global__ void k_shape_avg(int ncells, int nshape, int nper,
                            const double *__restrict__ in,
                            const double *__restrict__ w,
                            double *__restrict__ out) {
  const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= (int64_t)ncells * nper) {
    return;
  }
  const int64_t c = u / nper;
  const int j = (int)(u % nper);
  double acc = 0., norm = 0.;
  for (int s = 0; s < nshape; ++s) {
    acc += w[s] * in[(c * nshape + s) * nper + j];
    norm += w[s];
  }
  out[u] = acc * (1. / norm);
}

// --------------------------------------------------------- launchers -----

void tmx_launch_cg(int nmax, const int64_t *cg_off, double *cg, double *work,
                   int blocks, cudaStream_t stream) {
  k_cg<<<blocks, 128, 0, stream>>>(nmax, cg_off, cg, work);
}

void tmx_launch_orient_pairs(const TmxObsGrain *og, const int64_t *pstart,
                             const int32_t *order, int pmax, int64_t npairs,
                             const TmxMatSet &mats,
                             int nmat, const double *coeffs, int ncoef,
                             const int64_t *cg_off, const double *cg,
                             int cg_nmax, int mmax, int fold,
                             cudaStream_t stream) {
  if (npairs <= 0) {
    return;
  }
  const int wcap = 4 * (mmax + 1) + 2 * (2 * mmax + 1);
  const size_t smem = (size_t)8 * wcap * nmat * sizeof(double2);
  const int64_t want = (npairs + 7) / 8;
  const int blocks = (int)std::min<int64_t>(want, 148 * 8);
  if (nmat == 4 || nmat == 3) {
    // four warps per CTA: the matrices' buffers of 8 warps would leave room
    // for one CTA per SM
    const size_t smem4 = (size_t)4 * wcap * nmat * sizeof(double2);
    const int blocks4 = (int)std::min<int64_t>((npairs + 3) / 4, 148 * 16);
    if (nmat == 4) {
      cudaFuncSetAttribute(k_orient_pairs<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem4);
      k_orient_pairs<4><<<blocks4, 128, smem4, stream>>>(og, pstart, order, pmax, npairs,
                                                         mats, coeffs, ncoef, cg_off, cg,
                                                         cg_nmax, wcap, fold);
    } else {
      cudaFuncSetAttribute(k_orient_pairs<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem4);
      k_orient_pairs<3><<<blocks4, 128, smem4, stream>>>(og, pstart, order, pmax, npairs,
                                                         mats, coeffs, ncoef, cg_off, cg,
                                                         cg_nmax, wcap, fold);
    }
  } else {
    cudaFuncSetAttribute(k_orient_pairs<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    k_orient_pairs<1><<<blocks, 256, smem, stream>>>(og, pstart, order, pmax, npairs,
                                                     mats, coeffs, ncoef, cg_off, cg,
                                                     cg_nmax, wcap, fold);
  }
}

static size_t amp_smem(int nbmax, int nmat) {
  return (size_t)4 * nbmax * 32 * sizeof(double) +
         (size_t)nmat * 8 * 4 * 32 * sizeof(double2);
}

int tmx_amp_grid(int nbmax, int nmat) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (nmat == 4) {
    cudaFuncSetAttribute(k_amp<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)amp_smem(TMX_MAX_NB, 4));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_amp<4>, 256,
                                                  amp_smem(nbmax, 4));
  } else if (nmat == 3) {
    cudaFuncSetAttribute(k_amp<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)amp_smem(TMX_MAX_NB, 3));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_amp<3>, 256,
                                                  amp_smem(nbmax, 3));
  } else {
    cudaFuncSetAttribute(k_amp<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)amp_smem(TMX_MAX_NB, 1));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_amp<1>, 256,
                                                  amp_smem(nbmax, 1));
  }
  return std::max(1, sms * std::max(1, per_sm));
}

void tmx_launch_wigner_cols(const TmxAngle *angles, int nangles, int nmax,
                            double *pi, double *tau, cudaStream_t stream) {
  const int64_t n = (int64_t)nangles * (nmax + 1);
  if (n <= 0) {
    return;
  }
  k_wigner_cols<<<(int)((n + 127) / 128), 128, 0, stream>>>(angles, nangles, nmax,
                                                           pi, tau);
}

void tmx_launch_amp(const TmxAmpGroup *groups, int ngroups, const TmxSJob *jobs,
                    const TmxObsGrain *og, const TmxMatSet &mats, int nmat,
                    const TmxAngle *angles, const double2 *phis, double2 *xslot,
                    int nbmax, int grid, const double *wpi, const double *wtau,
                    int wnmax, cudaStream_t stream) {
  if (ngroups <= 0) {
    return;
  }
  const int blocks = std::min(grid, ngroups);
  if (nmat == 4) {
    k_amp<4><<<blocks, 256, amp_smem(nbmax, 4), stream>>>(groups, ngroups, jobs, og,
                                                          mats, angles, phis, xslot,
                                                          nbmax, wpi, wtau, wnmax);
  } else if (nmat == 3) {
    k_amp<3><<<blocks, 256, amp_smem(nbmax, 3), stream>>>(groups, ngroups, jobs, og,
                                                          mats, angles, phis, xslot,
                                                          nbmax, wpi, wtau, wnmax);
  } else {
    k_amp<1><<<blocks, 256, amp_smem(nbmax, 1), stream>>>(groups, ngroups, jobs, og,
                                                          mats, angles, phis, xslot,
                                                          nbmax, wpi, wtau, wnmax);
  }
}

void tmx_launch_q_epilogue(const TmxQJob *jobs, int njobs, const TmxObsGrain *og,
                           const double2 *S, const double *wts, int nacc,
                           double *qout, int qstride, int do_abs, int do_ext,
                           cudaStream_t stream) {
  if (njobs <= 0) {
    return;
  }
  k_q_epilogue<<<(njobs + 127) / 128, 128, 0, stream>>>(
      jobs, njobs, og, S, wts, nacc, qout, qstride, do_abs, do_ext);
}

void tmx_launch_dq_epilogue(const TmxQJob *jobs, int njobs,
                            const TmxObsGrain *og, const double2 *S,
                            const double2 *dSm, const double2 *dSr,
                            const double2 *dSd, double *dq, cudaStream_t stream) {
  if (njobs <= 0) {
    return;
  }
  k_dq_epilogue<<<(njobs + 127) / 128, 128, 0, stream>>>(jobs, njobs, og, S,
                                                         dSm, dSr, dSd, dq);
}

void tmx_launch_z_epilogue(int n, const double2 *S, double *zout,
                           cudaStream_t stream) {
  if (n <= 0) {
    return;
  }
  k_z_epilogue<<<(n + 127) / 128, 128, 0, stream>>>(n, S, zout);
}

void tmx_launch_shape_avg(int ncells, int nshape, int nper, const double *in,
                          const double *w, double *out, cudaStream_t stream) {
  const int64_t n = (int64_t)ncells * nper;
  if (n <= 0) {
    return;
  }
  k_shape_avg<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(ncells, nshape,
                                                               nper, in, w, out);
}
