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

__device__ static void orient_avg_grain(const TmxObsGrain G,
                                        const cplx *__restrict__ T,
                                        cplx *__restrict__ Ta,
                                        const double *__restrict__ coeffs,
                                        int ncoef,
                                        const int64_t *__restrict__ cg_off,
                                        const double *__restrict__ cg,
                                        int cg_nmax, cplx *S) {
  const int N = G.nmax;
  if (N <= 0 || G.coef_set < 0) {
    return; // disabled alignment: copied by the host
  }
  const double *p = coeffs + (int64_t)G.coef_set * ncoef;
  const cplx *Tg = T + G.t_off;
  cplx *Tag = Ta + G.t_off;
  for (int u = threadIdx.x; u < N * N; u += blockDim.x) {
    const int n1 = u / N + 1;
    const int n2 = u % N + 1;
    const int M = min(n1, n2);
    const int lo = abs(n1 - n2);
    const int hi = n1 + n2;
    const double *C = cg + cg_off[(n1 - 1) * cg_nmax + (n2 - 1)];
    // pass 1: S_a(N') = sum_m1 f(m1) (-1)^m1 CG(m1) T_m1(type a)
    for (int Np = lo; Np <= hi; ++Np) {
      const double *Cr = C + (int64_t)(Np - lo) * (M + 1);
      const bool even = ((Np + hi) % 2 == 0);
      const int i1a = 0, i2a = even ? 0 : 1;
      const int i1b = 1, i2b = even ? 1 : 0;
      cplx sa = mkc(0., 0.), sb = mkc(0., 0.);
      for (int m1 = 0; m1 <= M; ++m1) {
        const double f = ((m1 == 0) ? 1. : 2.) * ((m1 & 1) ? -1. : 1.) * Cr[m1];
        const cplx ta = Tg[telem(N, m1, i1a, n1, i2a, n2)];
        const cplx tb = Tg[telem(N, m1, i1b, n1, i2b, n2)];
        sa = cadd(sa, cscale(ta, f));
        sb = cadd(sb, cscale(tb, f));
      }
      S[2 * (Np - lo)] = sa;
      S[2 * (Np - lo) + 1] = sb;
    }
    // pass 2: Tavg_m = sum_N' p_N' (-1)^m CG(m) S(N')
    for (int m = 0; m <= M; ++m) {
      cplx e00 = mkc(0., 0.), e11 = e00, e01 = e00, e10 = e00;
      const double ms = (m & 1) ? -1. : 1.;
      for (int Np = lo; Np <= hi; ++Np) {
        const double f = ms * p[Np] * C[(int64_t)(Np - lo) * (M + 1) + m];
        const cplx sa = S[2 * (Np - lo)];
        const cplx sb = S[2 * (Np - lo) + 1];
        if ((Np + hi) % 2 == 0) {
          e00 = cadd(e00, cscale(sa, f));
          e11 = cadd(e11, cscale(sb, f));
        } else {
          e01 = cadd(e01, cscale(sa, f));
          e10 = cadd(e10, cscale(sb, f));
        }
      }
      Tag[telem(N, m, 0, n1, 0, n2)] = e00;
      Tag[telem(N, m, 1, n1, 1, n2)] = e11;
      Tag[telem(N, m, 0, n1, 1, n2)] = e01;
      Tag[telem(N, m, 1, n1, 0, n2)] = e10;
    }
  }
}


// Blocks stride over grains; threads over (n1, n2) of a grain. S[N'] (2
// complex per N') lives in a per-thread work slot of wstride elements.
__global__ void k_orient_avg(const TmxObsGrain *__restrict__ og, int ngrains,
                             const cplx *__restrict__ T, cplx *__restrict__ Ta,
                             const double *__restrict__ coeffs, int ncoef,
                             const int64_t *__restrict__ cg_off,
                             const double *__restrict__ cg, int cg_nmax,
                             cplx *__restrict__ work, int wstride) {
  cplx *S = work + ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * wstride;
  for (int gi = blockIdx.x; gi < ngrains; gi += gridDim.x) {
    orient_avg_grain(og[gi], T, Ta, coeffs, ncoef, cg_off, cg, cg_nmax, S);
  }
}

// -------------------------------------------------- forward amplitude ----

// d^n_{0m}(x) / sin x and d/dx for one m, n = 1..nmax
// (SpecialFunctions::wigner_dn_0m_sinx, SpecialFunctions.hpp:397-495)
__device__ static void wigner_sinx(double cosx, double sinx, double sinx_inv,
                                   int nmax, int m, double *y, double *dy) {
  if (fabs(1. - fabs(cosx)) <= 1.e-10) {
    if (m == 1) {
      int sign = 1;
      for (int n = 1; n < nmax + 1; ++n) {
        double dn = 0.5 * sqrt(n * (n + 1.));
        if (cosx < 0.) {
          dn *= sign;
        }
        y[n - 1] = dn;
        if (cosx < 0.) {
          dn = -dn;
        }
        dy[n - 1] = dn;
        sign = -sign;
      }
    } else {
      for (int i = 0; i < nmax; ++i) {
        y[i] = 0.;
        dy[i] = 0.;
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
      y[n] = d2 * sinx_inv;
      dy[n] = ddn;
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
    y[n] = 0.;
    dy[n] = 0.;
  }
  for (int n = m - 1; n < nmax; ++n) {
    const double np1 = n + 1.;
    const double np2 = n + 2.;
    const double np12p1 = 2. * np1 + 1.;
    const double s12 = sqrt(np1 * np1 - m2);
    const double s22 = sqrt(np2 * np2 - m2);
    const double dnp1 = (np12p1 * cosx * d2 - s12 * d1) / s22;
    const double ddn = sinx_inv * (np1 * s22 * dnp1 - np2 * s12 * d1) / np12p1;
    y[n] = d2 * sinx_inv;
    dy[n] = ddn;
    d1 = d2;
    d2 = dnp1;
  }
}

__device__ __forceinline__ double a_nn(int n1, int n2) {
  const double s1 = sqrt((2. * n1 + 1.) / ((n1 + 1.) * n1));
  const double s2 = sqrt((2. * n2 + 1.) / ((n2 + 1.) * n2));
  return s1 * s2;
}

// c_{n1 n2} = i^{n1 - n2 - 1} a_{n1 n2} (NBasedResources::get_cnn)
__device__ __forceinline__ cplx c_nn(int n1, int n2) {
  const double a = a_nn(n1, n2);
  switch ((((n1 - n2 - 1) % 4) + 4) % 4) {
  case 0:
    return mkc(a, 0.);
  case 1:
    return mkc(0., a);
  case 2:
    return mkc(-a, 0.);
  default:
    return mkc(0., -a);
  }
}

// One block per job (grain, theta_in, theta_out, azimuth list). Thread m
// forms X_m, the four (n, n') sums of order m without the azimuthal factor;
// then every azimuth p gets S = (1/k) sum_m (2 cos m phi, 2 sin m phi) X_m
// with e^{i m phi} built by repeated multiplication as in the reference.
__global__ void k_forward_s(const TmxSJob *__restrict__ jobs, int njobs,
                            const TmxObsGrain *__restrict__ og,
                            const cplx *__restrict__ Ta,
                            const TmxAngle *__restrict__ angles,
                            const cplx *__restrict__ phis,
                            cplx *__restrict__ S_out) {
  const int j = blockIdx.x;
  if (j >= njobs) {
    return;
  }
  const TmxSJob J = jobs[j];
  const TmxObsGrain G = og[J.grain];
  const int N = G.nmax;
  const cplx *T = Ta + G.t_off;
  __shared__ cplx X[TMX_MAX_NB + 2][4];
  const TmxAngle ai = angles[J.angle_in];
  const TmxAngle ao = angles[J.angle_out];
  double din[TMX_MAX_NB], ddin[TMX_MAX_NB], dout[TMX_MAX_NB], ddout[TMX_MAX_NB];
  for (int m = threadIdx.x; m <= N; m += blockDim.x) {
    wigner_sinx(ai.c, ai.s, ai.si, N, m, din, ddin);
    wigner_sinx(ao.c, ao.s, ao.si, N, m, dout, ddout);
    const int nmin = (m > 1) ? m : 1;
    cplx x0 = mkc(0., 0.), x1 = x0, x2 = x0, x3 = x0;
    for (int nn = nmin; nn < N + 1; ++nn) {
      const double pi_nn = m * din[nn - 1];
      const double tau_nn = ddin[nn - 1];
      for (int n = nmin; n < N + 1; ++n) {
        const double pi_n = m * dout[n - 1];
        const double tau_n = ddout[n - 1];
        const cplx c = c_nn(nn, n);
        const cplx T11 = T[telem(N, m, 0, n, 0, nn)];
        const cplx T22 = T[telem(N, m, 1, n, 1, nn)];
        if (m == 0) {
          const cplx f = cscale(cscale(c, tau_n), tau_nn);
          x0 = cadd(x0, cmul(f, T22));
          x3 = cadd(x3, cmul(f, T11));
        } else {
          const cplx T12 = T[telem(N, m, 0, n, 1, nn)];
          const cplx T21 = T[telem(N, m, 1, n, 0, nn)];
          const double pp = pi_n * pi_nn, pt = pi_n * tau_nn;
          const double tp = tau_n * pi_nn, tt = tau_n * tau_nn;
          const cplx s0 = cadd(cadd(cadd(cscale(T11, pp), cscale(T21, tp)),
                                    cscale(T12, pt)),
                               cscale(T22, tt));
          const cplx s1 = cadd(cadd(cadd(cscale(T11, pt), cscale(T21, tt)),
                                    cscale(T12, pp)),
                               cscale(T22, tp));
          const cplx s2 = cadd(cadd(cadd(cscale(T11, tp), cscale(T21, pp)),
                                    cscale(T12, tt)),
                               cscale(T22, pt));
          const cplx s3 = cadd(cadd(cadd(cscale(T11, tt), cscale(T21, pt)),
                                    cscale(T12, tp)),
                               cscale(T22, pp));
          x0 = cadd(x0, cmul(c, s0));
          x1 = cadd(x1, cmul(c, s1));
          x2 = cadd(x2, cmul(c, s2));
          x3 = cadd(x3, cmul(c, s3));
        }
      }
    }
    X[m][0] = x0;
    X[m][1] = x1;
    X[m][2] = x2;
    X[m][3] = x3;
  }
  __syncthreads();
  const double kinv = 1. / G.k;
  for (int p = threadIdx.x; p < J.nphi; p += blockDim.x) {
    const cplx e1 = phis[J.phi0 + p];
    cplx e = mkc(1., 0.);
    cplx s0 = mkc(0., 0.), s1 = s0, s2 = s0, s3 = s0;
    for (int m = 0; m <= N; ++m) {
      const double fcos = 2. * e.x;
      const double fsin = 2. * e.y;
      e = cmul(e, e1);
      if (m == 0) {
        s0 = cadd(s0, X[0][0]);
        s3 = cadd(s3, X[0][3]);
      } else {
        s0 = cadd(s0, cscale(X[m][0], fcos));
        s1 = cadd(s1, cscale(X[m][1], fsin));
        s2 = csub(s2, cscale(X[m][2], fsin));
        s3 = cadd(s3, cscale(X[m][3], fcos));
      }
    }
    cplx *o = S_out + (J.out + p) * 4;
    o[0] = cscale(s0, kinv);
    o[1] = cscale(s1, kinv);
    o[2] = cscale(s2, kinv);
    o[3] = cscale(s3, kinv);
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

void tmx_launch_orient_avg(const TmxObsGrain *og, int ngrains, const double2 *T,
                           double2 *Ta, const double *coeffs, int ncoef,
                           const int64_t *cg_off, const double *cg, int cg_nmax,
                           double2 *work, int wstride, int blocks, int threads,
                           cudaStream_t stream) {
  if (ngrains <= 0) {
    return;
  }
  k_orient_avg<<<blocks, threads, 0, stream>>>(og, ngrains, T, Ta, coeffs, ncoef,
                                               cg_off, cg, cg_nmax, work, wstride);
}

void tmx_launch_forward_s(const TmxSJob *jobs, int njobs, const TmxObsGrain *og,
                          const double2 *Ta, const TmxAngle *angles,
                          const double2 *phis, double2 *S, cudaStream_t stream) {
  if (njobs <= 0) {
    return;
  }
  k_forward_s<<<njobs, 128, 0, stream>>>(jobs, njobs, og, Ta, angles, phis, S);
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
