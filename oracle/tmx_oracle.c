/* CPU oracle for the CosTuuM T-matrix hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference's algorithms. Each function names the
 * reference file:line it follows (paths relative to the CosTuuM source tree)
 * and keeps the reference's operation order, so that the tables and blocks it
 * produces can be compared bit for bit with the reference build
 * (oracle/build_ref.sh). Built with -O2 -ffp-contract=off (no fused
 * multiply-add), like the reference's x86-64 build.
 *
 * This file is the checker for the CUDA path and never part of it: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 */
#include "tmx_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

#define CX(re, im) CMPLX((re), (im))

/* ------------------------------------------------------ Gauss-Legendre --- */

/* SpecialFunctions::get_gauss_legendre_points_and_weights,
 * src/SpecialFunctions.hpp:646-715 (Newton on P_n from the Lether-Wenston
 * initial guess; ascending nodes, symmetric fill) */
void or_gauss_legendre(int order, double *points, double *weights) {
  const unsigned ind = (unsigned)order % 2;
  const unsigned k = (unsigned)order / 2 + ind;
  for (unsigned i = 0; i < k; ++i) {
    const double theta_n_k = M_PI * (i + 0.75) / (order + 0.5);
    const double orderinv = 1. / order;
    const double orderinv2 = orderinv * orderinv;
    double x_i = (1. - 0.125 * orderinv2 + (5. / 38.) * orderinv * orderinv2 -
                  (2. / 25.) * orderinv2 * orderinv2 *
                      (1. - (14. / 39.) / (theta_n_k * theta_n_k))) *
                 cos(theta_n_k);
    unsigned niter = 0;
    double check = 1.e-16;
    double pa, pb;
    do {
      ++niter;
      if (niter > 100) {
        check *= 10.;
      }
      pb = 1.;
      double pc = x_i;
      for (unsigned j = 1; j < (unsigned)order; ++j) {
        pa = pb;
        pb = pc;
        pc = x_i * pb + (x_i * pb - pa) * j / (j + 1.);
      }
      pa = 1. / ((pb - x_i * pc) * order);
      pb = pa * pc * (1. - x_i * x_i);
      x_i = x_i - pb;
    } while (fabs(pb) > check * fabs(x_i));
    const unsigned m = order - i - 1;
    points[m] = x_i;
    weights[m] = 2. * pa * pa * (1. - x_i * x_i);
    if (i != k - 1 || ind != 1) {
      points[i] = -points[m];
      weights[i] = weights[m];
    }
  }
}

/* get_gauss_legendre_points_and_weights_ab, SpecialFunctions.hpp:737-751 */
void or_gauss_legendre_ab(int order, double a, double b, double *x,
                          double *w) {
  or_gauss_legendre(order, x, w);
  const double wfac = 0.5 * (b - a);
  const double xterm = 0.5 * (a + b);
  for (int i = 0; i < order; ++i) {
    x[i] = wfac * x[i] + xterm;
    w[i] *= wfac;
  }
}

/* gauss_legendre_quadrature, SpecialFunctions.hpp:771-810: increase the
 * order by one until either tolerance is met */
static double gl_quadrature(double (*f)(double, const void *), const void *args,
                            double lower, double upper, int start, int maximum,
                            double abs_tol, double rel_tol) {
  int order = start;
  double old_q = 0.;
  double absd = abs_tol + 1.;
  double reld = rel_tol + 1.;
  double *x = (double *)malloc(sizeof(double) * maximum);
  double *w = (double *)malloc(sizeof(double) * maximum);
  while (order < maximum && absd > abs_tol && reld > rel_tol) {
    or_gauss_legendre_ab(order, lower, upper, x, w);
    double new_q = 0.;
    for (int i = 0; i < order; ++i) {
      new_q += w[i] * f(x[i], args);
    }
    absd = fabs(new_q - old_q);
    reld = absd / fabs(new_q + old_q);
    old_q = new_q;
    ++order;
  }
  free(x);
  free(w);
  return old_q;
}

/* ------------------------------------------------------------- Bessel --- */

#define BESSEL_START 800 /* SPECIALFUNCTIONS_BESSEL_NMAX, :40 */

/* spherical_j_jdj_array, SpecialFunctions.hpp:201-240 (real argument):
 * downward ratio recurrence from n = 800, forward j_n = rho_n j_{n-1};
 * dj holds [z j_n(z)]' / z */
void or_bessel_j_real(int nmax, double z, double *j, double *dj) {
  or_bessel_j_real_start(nmax, BESSEL_START, z, j, dj);
}

/* the same recurrence started at an arbitrary index (for the start-index
 * equivalence tests) */
void or_bessel_j_real_start(int nmax, int start, double z, double *j,
                            double *dj) {
  double rho[BESSEL_START];
  const double zinv = 1. / z;
  const double twonp1 = 2. * start + 1.;
  rho[start - 1] = z / twonp1;
  for (unsigned i = 1; i < (unsigned)start; ++i) {
    const unsigned index = start - i;
    const double twoip1 = 2. * index + 1.;
    rho[index - 1] = 1. / (twoip1 * zinv - rho[index]);
  }
  const double j0 = sin(z) * zinv;
  j[0] = rho[0] * j0;
  dj[0] = j0 - j[0] * zinv;
  for (int i = 1; i < nmax; ++i) {
    j[i] = rho[i] * j[i - 1];
    const double ip1 = i + 1.;
    dj[i] = j[i - 1] - ip1 * zinv * j[i];
  }
}

/* same for a complex argument (std::complex arithmetic: every constant is a
 * complex number, so products and quotients are full complex operations) */
void or_bessel_j_complex(int nmax, double zr, double zi, double *jout,
                         double *djout) {
  or_bessel_j_complex_start(nmax, BESSEL_START, zr, zi, jout, djout);
}

void or_bessel_j_complex_start(int nmax, int start, double zr, double zi,
                               double *jout, double *djout) {
  cplx rho[BESSEL_START];
  const cplx z = CX(zr, zi);
  const cplx one = CX(1., 0.);
  const cplx zinv = one / z;
  const cplx twonp1 = CX(2. * start + 1., 0.);
  rho[start - 1] = z / twonp1;
  for (unsigned i = 1; i < (unsigned)start; ++i) {
    const unsigned index = start - i;
    const cplx twoip1 = CX(2. * index + 1., 0.);
    rho[index - 1] = one / (twoip1 * zinv - rho[index]);
  }
  const cplx j0 = csin(z) * zinv;
  cplx *j = (cplx *)jout;
  cplx *dj = (cplx *)djout;
  j[0] = rho[0] * j0;
  dj[0] = j0 - j[0] * zinv;
  for (int i = 1; i < nmax; ++i) {
    j[i] = rho[i] * j[i - 1];
    const cplx ip1 = CX(i + 1., 0.);
    dj[i] = j[i - 1] - ip1 * zinv * j[i];
  }
}

/* spherical_y_ydy_array, SpecialFunctions.hpp:106-140 (real argument):
 * y_1, y_2 in closed form, then the upward recurrence */
void or_bessel_y_real(int nmax, double z, double *y, double *dy) {
  const double cosz = cos(z);
  const double sinz = sin(z);
  const double zinv = 1. / z;
  const double zinv2 = zinv * zinv;
  const double zinv3 = zinv2 * zinv;
  y[0] = -cosz * zinv2 - sinz * zinv;
  y[1] = (-3. * zinv3 + zinv) * cosz - 3. * zinv2 * sinz;
  dy[0] = -zinv * (cosz + y[0]);
  dy[1] = y[0] - 2. * zinv * y[1];
  for (int i = 2; i < nmax; ++i) {
    const double twoip1 = 2. * i + 1.;
    const double ip1 = i + 1.;
    y[i] = twoip1 * zinv * y[i - 1] - y[i - 2];
    dy[i] = y[i - 1] - ip1 * zinv * y[i];
  }
}

/* ------------------------------------------------------------ Wigner d --- */

/* wigner_dn_0m, SpecialFunctions.hpp:302-371: d^n_{0m}(x) and d/dx for
 * n = 1 .. nmax by forward recurrence in n */
void or_wigner_d(double cosx, int nmax, int m, double *y, double *dy) {
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
      y[n] = d2;
      dy[n] = ddn;
      d1 = d2;
      d2 = dnp1;
    }
  } else {
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
      const double sqrtnp12mm2 = sqrt(np1 * np1 - m2);
      const double sqrtnp22mm2 = sqrt(np2 * np2 - m2);
      const double dnp1 = (np12p1 * cosx * d2 - sqrtnp12mm2 * d1) / sqrtnp22mm2;
      const double ddn =
          sinxinv * (np1 * sqrtnp22mm2 * dnp1 - np2 * sqrtnp12mm2 * d1) /
          np12p1;
      y[n] = d2;
      dy[n] = ddn;
      d1 = d2;
      d2 = dnp1;
    }
  }
}

/* wigner_dn_0m_sinx, SpecialFunctions.hpp:397-495: d^n_{0m}/sin x, with the
 * |cos x| -> 1 limit handled explicitly */
void or_wigner_d_sinx(double cosx, double sinx, double sinx_inv, int nmax,
                      int m, double *y, double *dy) {
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
  } else {
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
      const double sqrtnp12mm2 = sqrt(np1 * np1 - m2);
      const double sqrtnp22mm2 = sqrt(np2 * np2 - m2);
      const double dnp1 = (np12p1 * cosx * d2 - sqrtnp12mm2 * d1) / sqrtnp22mm2;
      const double ddn =
          sinx_inv * (np1 * sqrtnp22mm2 * dnp1 - np2 * sqrtnp12mm2 * d1) /
          np12p1;
      y[n] = d2 * sinx_inv;
      dy[n] = ddn;
      d1 = d2;
      d2 = dnp1;
    }
  }
}

/* get_equal_volume_to_equal_surface_area_sphere_ratio,
 * SpecialFunctions.hpp:557-583 */
double or_rv_over_rs(double d) {
  if (d > 1.) {
    const double d2 = d * d;
    const double e = sqrt(1. - 1. / d2);
    const double cbrtd2 = cbrt(d2);
    return 1. / sqrt(0.25 * (2. * cbrtd2 +
                             log((1. + e) / (1. - e)) / (e * cbrtd2 * cbrtd2)));
  } else if (d < 1.) {
    const double cbrtd = cbrt(d);
    const double e = sqrt(1. - d * d);
    return 1. / sqrt(0.5 * (cbrtd * cbrtd + asin(e) / (e * cbrtd)));
  }
  return 1.;
}

/* ------------------------------------------------------ Clebsch-Gordan --- */

/* get_clebsch_gordan_coefficients, SpecialFunctions.hpp:1131-1244: the row
 * <n1 m1 n2 -m1 | N 0> for m1 = -min(n1,n2) .. min(n1,n2), by the upper-row
 * ladder recursion (normalised) followed by the M-lowering recursion */
int or_clebsch_gordan_row(int n1, int n2, int N, double *out) {
  const int nsize = 2 * n1 + 1;
  double *C = (double *)calloc((size_t)(N + 1) * nsize, sizeof(double));
  C[N * nsize + n1 + n1] = 1.;
  double norm = 1.;
  const int lo = (-n1 > N - n2 - 1) ? -n1 : N - n2 - 1;
  for (int m1t = n1 - 1; m1t >= lo; --m1t) {
    const double cplus_n2m2 = sqrt((n2 - N + m1t + 1.) * (n2 + N - m1t));
    const double cplus_n1m1m1 = sqrt((n1 - m1t) * (n1 + m1t + 1.));
    const double c_n1m1p1 = C[N * nsize + m1t + 1 + n1];
    const double cnext = -cplus_n2m2 * c_n1m1p1 / cplus_n1m1m1;
    C[N * nsize + m1t + n1] = cnext;
    norm += cnext * cnext;
  }
  const double inverse_norm = 1. / sqrt(norm);
  for (int m1t = n1; m1t >= lo; --m1t) {
    C[N * nsize + m1t + n1] *= inverse_norm;
  }
  for (int Mt = N - 1; Mt >= 0; --Mt) {
    const double cmin_inverse = 1. / sqrt((N + Mt + 1.) * (N - Mt));
    const int a = (-n1 > Mt - n2) ? -n1 : Mt - n2;
    const int b = (n1 < Mt + n2) ? n1 : Mt + n2;
    for (int m1t = a; m1t <= b; ++m1t) {
      const int m2t = Mt - m1t;
      double term1 = 0.;
      if (m1t + 1 <= n1) {
        const double cmin_n1m1p1 = sqrt((n1 + m1t + 1.) * (n1 - m1t));
        term1 = cmin_n1m1p1 * C[(Mt + 1) * nsize + m1t + 1 + n1];
      }
      double term2 = 0.;
      if (m2t + 1 <= n2) {
        const double cmin_n2m2p1 = sqrt((n2 + m2t + 1.) * (n2 - m2t));
        term2 = cmin_n2m2p1 * C[(Mt + 1) * nsize + m1t + n1];
      }
      C[Mt * nsize + m1t + n1] = cmin_inverse * (term1 + term2);
    }
  }
  const int nmin = (n1 < n2) ? n1 : n2;
  for (int i = 0; i < 2 * nmin + 1; ++i) {
    out[i] = C[i - nmin + n1];
  }
  free(C);
  return 2 * nmin + 1;
}

/* -------------------------------------------------------- plu_inverse --- */

/* Matrix::plu_inverse, src/Matrix.hpp:261-384: Doolittle LU with partial
 * pivoting on max |A_ji|, U^-1 by substitution, inv(A) L = U^-1, and the
 * final column exchanges in reverse pivot order. A is n x n with leading
 * dimension lda (complex elements). */
static void plu_inverse_ld(int n, int lda, cplx *A, int *pivot, cplx *work) {
#define EL(i, j) A[(size_t)(i) * lda + (j)]
  const cplx one = CX(1., 0.);
  for (int i = 0; i < n; ++i) {
    int imax = i;
    double smax = cabs(EL(imax, i));
    for (int j = i + 1; j < n; ++j) {
      const double s = cabs(EL(j, i));
      if (s > smax) {
        smax = s;
        imax = j;
      }
    }
    pivot[i] = imax;
    if (i != imax) {
      for (int j = 0; j < n; ++j) {
        const cplx t = EL(i, j);
        EL(i, j) = EL(imax, j);
        EL(imax, j) = t;
      }
    }
    const cplx aii_inv = one / EL(i, i);
    for (int j = i + 1; j < n; ++j) {
      EL(j, i) *= aii_inv;
    }
    for (int j = i + 1; j < n; ++j) {
      for (int k = i + 1; k < n; ++k) {
        EL(j, k) -= EL(j, i) * EL(i, k);
      }
    }
  }
  for (int i = 0; i < n; ++i) {
    EL(i, i) = one / EL(i, i);
    for (int j = i + 1; j < n; ++j) {
      cplx aij = CX(0., 0.);
      for (int k = i; k < j; ++k) {
        aij -= EL(i, k) * EL(k, j);
      }
      EL(i, j) = aij / EL(j, j);
    }
  }
  for (int jp1 = n; jp1 > 0; --jp1) {
    const int j = jp1 - 1;
    for (int i = 0; i < jp1; ++i) {
      work[i] = EL(i, j);
    }
    for (int i = jp1; i < n; ++i) {
      work[i] = CX(0., 0.);
    }
    for (int k = jp1; k < n; ++k) {
      for (int i = 0; i < n; ++i) {
        work[i] -= EL(i, k) * EL(k, j);
      }
    }
    for (int i = 0; i < n; ++i) {
      EL(i, j) = work[i];
    }
  }
  for (int jp1 = n; jp1 > 0; --jp1) {
    const int j = jp1 - 1;
    const int jp = pivot[j];
    if (jp != j) {
      for (int i = 0; i < n; ++i) {
        const cplx t = EL(i, j);
        EL(i, j) = EL(i, jp);
        EL(i, jp) = t;
      }
    }
  }
#undef EL
}

void or_plu_inverse(int n, double *a) {
  int *pivot = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  cplx *work = (cplx *)malloc(sizeof(cplx) * (n > 0 ? n : 1));
  plu_inverse_ld(n, n, (cplx *)a, pivot, work);
  free(pivot);
  free(work);
}

/* ------------------------------------------- orientation distributions --- */

struct od_args {
  int kind;
  double norm;
  int order;
};

/* OrientationDistribution::operator() for the random distribution is the
 * constant 1/2 (OrientationDistribution.hpp:63-66) */
static double od_p(double beta) {
  (void)beta;
  return 0.5;
}

static double od_norm_integrand(double beta, const void *a) {
  (void)a;
  const double sinbeta = sin(beta);
  return sinbeta * od_p(beta);
}

static double od_coeff_integrand(double beta, const void *vargs) {
  const struct od_args *args = (const struct od_args *)vargs;
  const double cosbeta = cos(beta);
  const double sinbeta = sin(beta);
  double dn;
  if (args->order > 0) {
    double *d = (double *)malloc(sizeof(double) * args->order);
    double *dd = (double *)malloc(sizeof(double) * args->order);
    or_wigner_d(cosbeta, args->order, 0, d, dd);
    dn = d[args->order - 1];
    free(d);
    free(dd);
  } else {
    dn = 1.;
  }
  const double pbeta = args->norm * od_p(beta);
  return sinbeta * pbeta * dn;
}

/* OrientationDistribution::initialise (OrientationDistribution.hpp:220-243),
 * MishchenkoOrientationDistribution (MishchenkoOrientationDistribution.hpp:
 * 107-118) and DavisGreensteinOrientationDistribution
 * (DavisGreensteinOrientationDistribution.hpp:81-102) */
void or_orientation_coefficients(int kind, double param, int order,
                                 double *out) {
  for (int i = 0; i <= order; ++i) {
    out[i] = 0.;
  }
  if (kind == 0) {
    struct od_args a = {0, 1., 0};
    const double norm =
        gl_quadrature(od_norm_integrand, &a, 0., M_PI, 100, 1000, 1.e-10,
                      1.e-5);
    a.norm = 1. / norm;
    out[0] = 1.;
    for (int i = 1; i <= order; ++i) {
      a.order = i;
      out[i] = gl_quadrature(od_coeff_integrand, &a, 0., M_PI, 2 * (i + 1),
                             100 * (i + 1), 1.e-10, 1.e-5);
    }
  } else if (kind == 1) {
    out[0] = 1.;
    if (order >= 2) {
      out[2] = 1.5 * param - 0.5;
    }
  } else {
    if (param < 1.) {
      double nominator = 1.;
      double denominator = 2.;
      out[0] = 1.;
      for (int i = 1; 2 * i < order + 1; ++i) {
        const int sign = (i % 2 == 0) ? 1 : -1;
        out[2 * i] = sign * nominator / denominator;
        nominator *= 2. * i + 1.;
        denominator *= 2. * (i + 1.);
      }
    } else {
      for (int i = 0; i <= order; ++i) {
        out[i] = 1.;
      }
    }
  }
}

/* ----------------------------------------------------- T-matrix blocks --- */

long or_tmatrix_block_offset(int nmax, int m) {
  long off = 0;
  for (int mm = 0; mm < m; ++mm) {
    const long nb = (mm == 0) ? nmax : nmax + 1 - mm;
    off += 2 * 4 * nb * nb;
  }
  return off;
}

long or_tmatrix_size(int nmax) { return or_tmatrix_block_offset(nmax, nmax + 1); }

/* the per-order tables of one grain: GaussBasedResources::execute
 * (GaussBasedResources.hpp:132-152), get_r_dr_spheroid
 * (SpecialFunctions.hpp:872-893), ParticleGeometryResource::execute
 * (ParticleGeometryResource.hpp:135-149), InteractionVariables
 * (InteractionResource.hpp:50-132), InteractionTask::execute
 * (InteractionResource.hpp:478-527), NBasedResources::execute
 * (NBasedResources.hpp:115-137) */
struct tables {
  int nmax, ngauss;
  double k, k2;
  cplx kmr, k2mr;
  double *costheta, *weight, *sinthetainv, *sintheta2inv;
  double *r, *r2, *drr;
  double *kr, *krinv;
  cplx *krmr, *krmrinv;
  double *jkr, *ykr, *djkr, *dykr; /* [2 ngauss][nmax] */
  cplx *jkrmr, *djkrmr;
};

static void tables_build(struct tables *t, double r_ev, double wavelength,
                         double mr, double mi, double axis_ratio, int nmax,
                         int ngauss) {
  const int n2g = 2 * ngauss;
  t->nmax = nmax;
  t->ngauss = ngauss;
  t->costheta = (double *)calloc(n2g, sizeof(double));
  t->weight = (double *)calloc(n2g, sizeof(double));
  t->sinthetainv = (double *)calloc(n2g, sizeof(double));
  t->sintheta2inv = (double *)calloc(n2g, sizeof(double));
  t->r = (double *)calloc(n2g, sizeof(double));
  t->r2 = (double *)calloc(n2g, sizeof(double));
  t->drr = (double *)calloc(n2g, sizeof(double));
  t->kr = (double *)calloc(n2g, sizeof(double));
  t->krinv = (double *)calloc(n2g, sizeof(double));
  t->krmr = (cplx *)calloc(n2g, sizeof(cplx));
  t->krmrinv = (cplx *)calloc(n2g, sizeof(cplx));
  t->jkr = (double *)calloc((size_t)n2g * nmax, sizeof(double));
  t->ykr = (double *)calloc((size_t)n2g * nmax, sizeof(double));
  t->djkr = (double *)calloc((size_t)n2g * nmax, sizeof(double));
  t->dykr = (double *)calloc((size_t)n2g * nmax, sizeof(double));
  t->jkrmr = (cplx *)calloc((size_t)n2g * nmax, sizeof(cplx));
  t->djkrmr = (cplx *)calloc((size_t)n2g * nmax, sizeof(cplx));

  or_gauss_legendre(n2g, t->costheta, t->weight);
  for (int ig = 0; ig < ngauss; ++ig) {
    const double s2i =
        1. / ((1. - t->costheta[ig]) * (1. + t->costheta[ig]));
    t->sintheta2inv[ig] = s2i;
    t->sintheta2inv[n2g - ig - 1] = s2i;
    const double si = sqrt(s2i);
    t->sinthetainv[ig] = si;
    t->sinthetainv[n2g - ig - 1] = si;
  }
  {
    const double a = cbrt(axis_ratio);
    const double a2 = a * a;
    const double d2 = axis_ratio * axis_ratio;
    const double d2m1 = d2 - 1.;
    for (int i = 0; i < n2g / 2; ++i) {
      const double c2 = t->costheta[i] * t->costheta[i];
      const double s2 = (1. - t->costheta[i]) * (1. + t->costheta[i]);
      const double s = sqrt(s2);
      const double r2oa2 = 1. / (s2 + d2 * c2);
      t->r2[i] = a2 * r2oa2;
      t->r2[n2g - i - 1] = t->r2[i];
      t->drr[i] = r2oa2 * t->costheta[i] * s * d2m1;
      t->drr[n2g - i - 1] = -t->drr[i];
    }
    for (int i = 0; i < n2g; ++i) {
      t->r[i] = sqrt(t->r2[i]);
    }
  }
  const cplx m = CX(mr, mi);
  t->k = 2. * M_PI / wavelength;
  t->k2 = t->k * t->k;
  t->kmr = m * t->k;
  t->k2mr = m * t->k2;
  for (int ig = 0; ig < n2g; ++ig) {
    t->kr[ig] = t->k * t->r[ig] * r_ev;
    t->krmr[ig] = t->kmr * t->r[ig] * r_ev;
    t->krinv[ig] = 1. / t->kr[ig];
    t->krmrinv[ig] = CX(1., 0.) / t->krmr[ig];
  }
  for (int ig = 0; ig < n2g; ++ig) {
    or_bessel_j_real(nmax, t->kr[ig], t->jkr + (size_t)ig * nmax,
                     t->djkr + (size_t)ig * nmax);
    or_bessel_y_real(nmax, t->kr[ig], t->ykr + (size_t)ig * nmax,
                     t->dykr + (size_t)ig * nmax);
    or_bessel_j_complex(nmax, creal(t->krmr[ig]), cimag(t->krmr[ig]),
                        (double *)(t->jkrmr + (size_t)ig * nmax),
                        (double *)(t->djkrmr + (size_t)ig * nmax));
  }
}

static void tables_free(struct tables *t) {
  free(t->costheta);
  free(t->weight);
  free(t->sinthetainv);
  free(t->sintheta2inv);
  free(t->r);
  free(t->r2);
  free(t->drr);
  free(t->kr);
  free(t->krinv);
  free(t->krmr);
  free(t->krmrinv);
  free(t->jkr);
  free(t->ykr);
  free(t->djkr);
  free(t->dykr);
  free(t->jkrmr);
  free(t->djkrmr);
}

/* a_{n1 n2} = sqrt((2n1+1)/(n1(n1+1))) sqrt((2n2+1)/(n2(n2+1)))
 * (NBasedResources.hpp:115-137) */
static double ann(int n1, int n2) {
  const double nn1 = (n1 + 1.) * (double)n1;
  const double nn2 = (n2 + 1.) * (double)n2;
  const double s1 = sqrt((2. * n1 + 1.) / nn1);
  const double s2 = sqrt((2. * n2 + 1.) / nn2);
  return s1 * s2;
}

/* c_{n1 n2} = i^{n1 - n2 - 1} a_{n1 n2} (NBasedResources::get_cnn) */
static cplx cnn(int n1, int n2) {
  const double a = ann(n1, n2);
  const int p = (((n1 - n2 - 1) % 4) + 4) % 4;
  switch (p) {
  case 0:
    return CX(a, 0.);
  case 1:
    return CX(0., a);
  case 2:
    return CX(-a, 0.);
  default:
    return CX(0., -a);
  }
}

/* WignerDResources::execute / get_wigner_functions
 * (WignerDResources.hpp:147-174, 232-247): for orders below 100 the
 * functions at the lower-half node ig are the mirrored values of the
 * upper-half node 2 ngauss - 1 - ig, with signs (-1)^n and -(-1)^n; at
 * order >= 100 they are evaluated directly at node ig */
static void wigner_at_node(const struct tables *t, int m, int ig, double *d,
                           double *dd) {
  const int order = t->nmax;
  const int n2g = 2 * t->ngauss;
  if (order < 100) {
    const int iu = n2g - 1 - ig;
    or_wigner_d(t->costheta[iu], order, m, d, dd);
    int sign = 1;
    for (int n = 0; n < order; ++n) {
      sign = -sign;
      d[n] = sign * d[n];
      dd[n] = -sign * dd[n];
    }
  } else {
    or_wigner_d(t->costheta[ig], order, m, d, dd);
  }
}

/* assembly of the Q and RgQ blocks for one m (TMatrixM0Task::execute,
 * TMatrixResource.hpp:601-709 for m = 0; TMatrixMAllTask::execute,
 * TMatrixResource.hpp:934-1100 for m >= 1). Q and RgQ are 2nb x 2nb. */
static void assemble(const struct tables *t, int m, cplx *Q, cplx *RgQ) {
  const int nmax = t->nmax;
  const int ngauss = t->ngauss;
  const double k2 = t->k2;
  const cplx k2mr = t->k2mr;
  double *wd = (double *)malloc(sizeof(double) * nmax);
  double *dwd = (double *)malloc(sizeof(double) * nmax);
  if (m == 0) {
    const int n2 = 2 * nmax;
    memset(Q, 0, sizeof(cplx) * n2 * n2);
    memset(RgQ, 0, sizeof(cplx) * n2 * n2);
#define QE(M, i, j) M[(size_t)(i) * n2 + (j)]
    for (int ig = 1; ig < ngauss + 1; ++ig) {
      wigner_at_node(t, 0, ig - 1, wd, dwd);
      for (int n1 = 1; n1 < nmax + 1; ++n1) {
        const double n1n1p1 = n1 * (n1 + 1.);
        const int i1 = n1;
        const int ii1 = i1 + nmax;
        for (int nn2 = 1; nn2 < nmax + 1; ++nn2) {
          const double n2n2p1 = nn2 * (nn2 + 1.);
          const int i2 = nn2;
          const int ii2 = i2 + nmax;
          if ((n1 + nn2) % 2 == 0) {
            const int g = ig - 1;
            const double wigner_n1 = wd[n1 - 1];
            const double dwigner_n1 = dwd[n1 - 1];
            const double wigner_n2 = wd[nn2 - 1];
            const double dwigner_n2 = dwd[nn2 - 1];
            const double wn1dwn2 = wigner_n1 * dwigner_n2;
            const double dwn1wn2 = dwigner_n1 * wigner_n2;
            const double dwn1dwn2 = dwigner_n1 * dwigner_n2;
            const double jkrn1 = t->jkr[(size_t)g * nmax + n1 - 1];
            const double ykrn1 = t->ykr[(size_t)g * nmax + n1 - 1];
            const cplx hkrn1 = CX(jkrn1, ykrn1);
            const double djkrn1 = t->djkr[(size_t)g * nmax + n1 - 1];
            const double dykrn1 = t->dykr[(size_t)g * nmax + n1 - 1];
            const cplx dhkrn1 = CX(djkrn1, dykrn1);
            const cplx jkrmrn2 = t->jkrmr[(size_t)g * nmax + nn2 - 1];
            const cplx djkrmrn2 = t->djkrmr[(size_t)g * nmax + nn2 - 1];
            const cplx c1 = jkrmrn2 * jkrn1;
            const cplx b1 = jkrmrn2 * hkrn1;
            const cplx c2 = jkrmrn2 * djkrn1;
            const cplx b2 = jkrmrn2 * dhkrn1;
            const double krinvi = t->krinv[g];
            const cplx c3 = krinvi * c1;
            const cplx b3 = krinvi * b1;
            const cplx c4 = jkrn1 * djkrmrn2;
            const cplx b4 = hkrn1 * djkrmrn2;
            const cplx krmrinvi = t->krmrinv[g];
            const cplx c5 = c1 * krmrinvi;
            const cplx b5 = b1 * krmrinvi;
            const double wr2i = t->weight[g] * t->r2[g];
            const double dr_over_ri = t->drr[g];
            const double an12 = ann(n1, nn2);
            const double f1 = wr2i * dwn1dwn2;
            const double f2 = wr2i * dr_over_ri * n1n1p1 * wn1dwn2;
            const cplx this_J12 = -an12 * (f1 * b2 + f2 * b3);
            const cplx this_RgJ12 = -an12 * (f1 * c2 + f2 * c3);
            const double f3 = wr2i * dr_over_ri * n2n2p1 * dwn1wn2;
            const cplx this_J21 = an12 * (f1 * b4 + f3 * b5);
            const cplx this_RgJ21 = an12 * (f1 * c4 + f3 * c5);
            QE(Q, i1 - 1, i2 - 1) += k2mr * this_J21 + k2 * this_J12;
            QE(RgQ, i1 - 1, i2 - 1) += k2mr * this_RgJ21 + k2 * this_RgJ12;
            QE(Q, ii1 - 1, ii2 - 1) += k2mr * this_J12 + k2 * this_J21;
            QE(RgQ, ii1 - 1, ii2 - 1) += k2mr * this_RgJ12 + k2 * this_RgJ21;
          }
        }
      }
    }
#undef QE
  } else {
    const double m2 = (double)(m * m);
    const int nm = nmax + 1 - m;
    const int nm2 = 2 * nm;
    const cplx icompl = CX(0., 1.);
    memset(Q, 0, sizeof(cplx) * nm2 * nm2);
    memset(RgQ, 0, sizeof(cplx) * nm2 * nm2);
#define QE(M, i, j) M[(size_t)(i) * nm2 + (j)]
    for (int ig = 0; ig < ngauss; ++ig) {
      wigner_at_node(t, m, ig, wd, dwd);
      for (int n1 = m; n1 < nmax + 1; ++n1) {
        const double n1n1p1 = n1 * (n1 + 1.);
        const int i1 = n1 + 1 - m;
        const int ii1 = i1 + nm;
        for (int nn2 = m; nn2 < nmax + 1; ++nn2) {
          const double n2n2p1 = nn2 * (nn2 + 1.);
          const int i2 = nn2 + 1 - m;
          const int ii2 = i2 + nm;
          const int sign = ((n1 + nn2) % 2 == 0) ? 1 : -1;
          const double wigner_n1 = wd[n1 - 1];
          const double dwigner_n1 = dwd[n1 - 1];
          const double wigner_n2 = wd[nn2 - 1];
          const double dwigner_n2 = dwd[nn2 - 1];
          const double wn1wn2 = wigner_n1 * wigner_n2;
          const double wn1dwn2 = wigner_n1 * dwigner_n2;
          const double dwn1wn2 = dwigner_n1 * wigner_n2;
          const double jkrn1 = t->jkr[(size_t)ig * nmax + n1 - 1];
          const double ykrn1 = t->ykr[(size_t)ig * nmax + n1 - 1];
          const cplx hkrn1 = CX(jkrn1, ykrn1);
          const double djkrn1 = t->djkr[(size_t)ig * nmax + n1 - 1];
          const double dykrn1 = t->dykr[(size_t)ig * nmax + n1 - 1];
          const cplx dhkrn1 = CX(djkrn1, dykrn1);
          const cplx jkrmrn2 = t->jkrmr[(size_t)ig * nmax + nn2 - 1];
          const cplx djkrmrn2 = t->djkrmr[(size_t)ig * nmax + nn2 - 1];
          const cplx c1 = jkrmrn2 * jkrn1;
          const cplx b1 = jkrmrn2 * hkrn1;
          const cplx c2 = jkrmrn2 * djkrn1;
          const cplx b2 = jkrmrn2 * dhkrn1;
          const double krinvi = t->krinv[ig];
          const cplx c4 = djkrmrn2 * jkrn1;
          const cplx b4 = djkrmrn2 * hkrn1;
          const cplx krmrinvi = t->krmrinv[ig];
          const double dr_over_ri = t->drr[ig];
          const double an12 = ann(n1, nn2);
          if (sign < 0) {
            const double dsi =
                t->sinthetainv[ig] * m * t->weight[ig] * t->r2[ig];
            const cplx c6 = djkrmrn2 * djkrn1;
            const cplx b6 = djkrmrn2 * dhkrn1;
            const cplx c7 = c4 * krinvi;
            const cplx b7 = b4 * krinvi;
            const cplx c8 = c2 * krmrinvi;
            const cplx b8 = b2 * krmrinvi;
            const double e1 = dsi * (wn1dwn2 + dwn1wn2);
            const cplx this_J11 = icompl * an12 * (e1 * b1);
            const cplx this_RgJ11 = icompl * an12 * (e1 * c1);
            const double factor = dsi * dr_over_ri * wn1wn2;
            const double e2 = factor * n1n1p1;
            const double e3 = factor * n2n2p1;
            const cplx this_J22 = icompl * an12 * (e1 * b6 + e2 * b7 + e3 * b8);
            const cplx this_RgJ22 =
                icompl * an12 * (e1 * c6 + e2 * c7 + e3 * c8);
            QE(Q, i1 - 1, ii2 - 1) += k2mr * this_J11 + k2 * this_J22;
            QE(RgQ, i1 - 1, ii2 - 1) += k2mr * this_RgJ11 + k2 * this_RgJ22;
            QE(Q, ii1 - 1, i2 - 1) += k2mr * this_J22 + k2 * this_J11;
            QE(RgQ, ii1 - 1, i2 - 1) += k2mr * this_RgJ22 + k2 * this_RgJ11;
          } else {
            const double wr2i = t->weight[ig] * t->r2[ig];
            const double dssi = t->sintheta2inv[ig] * m2;
            const cplx c3 = krinvi * c1;
            const cplx b3 = krinvi * b1;
            const cplx c5 = c1 * krmrinvi;
            const cplx b5 = b1 * krmrinvi;
            const double f1 = wr2i * (wn1wn2 * dssi + dwigner_n1 * dwigner_n2);
            const double f2 = wr2i * dr_over_ri * n1n1p1 * wn1dwn2;
            const cplx this_J12 = -an12 * (f1 * b2 + f2 * b3);
            const cplx this_RgJ12 = -an12 * (f1 * c2 + f2 * c3);
            const double f3 = wr2i * dr_over_ri * n2n2p1 * dwn1wn2;
            const cplx this_J21 = an12 * (f1 * b4 + f3 * b5);
            const cplx this_RgJ21 = an12 * (f1 * c4 + f3 * c5);
            QE(Q, i1 - 1, i2 - 1) += k2mr * this_J21 + k2 * this_J12;
            QE(RgQ, i1 - 1, i2 - 1) += k2mr * this_RgJ21 + k2 * this_RgJ12;
            QE(Q, ii1 - 1, ii2 - 1) += k2mr * this_J12 + k2 * this_J21;
            QE(RgQ, ii1 - 1, ii2 - 1) += k2mr * this_RgJ12 + k2 * this_RgJ21;
          }
        }
      }
    }
#undef QE
  }
  free(wd);
  free(dwd);
}

/* T = -RgQ Q^-1 with the explicit inverse (TMatrixResource.hpp:712-730,
 * 1102-1119) */
static void form_t(int nb, cplx *Q, const cplx *RgQ, cplx *T) {
  const int n2 = 2 * nb;
  int *pivot = (int *)malloc(sizeof(int) * n2);
  cplx *work = (cplx *)malloc(sizeof(cplx) * n2);
  plu_inverse_ld(n2, n2, Q, pivot, work);
  for (int i = 0; i < nb; ++i) {
    for (int j = 0; j < nb; ++j) {
      cplx t00 = CX(0., 0.), t10 = CX(0., 0.), t01 = CX(0., 0.),
           t11 = CX(0., 0.);
      for (int k = 0; k < n2; ++k) {
        t00 -= RgQ[(size_t)i * n2 + k] * Q[(size_t)k * n2 + j];
        t10 -= RgQ[(size_t)(nb + i) * n2 + k] * Q[(size_t)k * n2 + j];
        t01 -= RgQ[(size_t)i * n2 + k] * Q[(size_t)k * n2 + nb + j];
        t11 -= RgQ[(size_t)(nb + i) * n2 + k] * Q[(size_t)k * n2 + nb + j];
      }
      T[(size_t)i * n2 + j] = t00;
      T[(size_t)(nb + i) * n2 + j] = t10;
      T[(size_t)i * n2 + nb + j] = t01;
      T[(size_t)(nb + i) * n2 + nb + j] = t11;
    }
  }
  free(pivot);
  free(work);
}

/* m = 0 sums (TMatrixResource.hpp:743-756) */
static void m0_sums(int nmax, const cplx *T0, double *qsca, double *qext) {
  const int n2 = 2 * nmax;
  double qs = 0., qe = 0.;
  for (int n = 1; n < nmax + 1; ++n) {
    const double dn1 = 2. * n + 1.;
    const cplx a = T0[(size_t)(n - 1) * n2 + n - 1];
    const cplx b = T0[(size_t)(nmax + n - 1) * n2 + nmax + n - 1];
    const double na = creal(a) * creal(a) + cimag(a) * cimag(a);
    const double nb = creal(b) * creal(b) + cimag(b) * cimag(b);
    qs += dn1 * (na + nb);
    qe += dn1 * (creal(a) + creal(b));
  }
  *qsca = qs;
  *qext = qe;
}

void or_tmatrix_m0(double r_ev, double wavelength, double mr, double mi,
                   double axis_ratio, int nmax, int ngauss, double *T0,
                   double *qsca, double *qext) {
  struct tables t;
  tables_build(&t, r_ev, wavelength, mr, mi, axis_ratio, nmax, ngauss);
  const int n2 = 2 * nmax;
  cplx *Q = (cplx *)malloc(sizeof(cplx) * n2 * n2);
  cplx *RgQ = (cplx *)malloc(sizeof(cplx) * n2 * n2);
  assemble(&t, 0, Q, RgQ);
  form_t(nmax, Q, RgQ, (cplx *)T0);
  m0_sums(nmax, (const cplx *)T0, qsca, qext);
  free(Q);
  free(RgQ);
  tables_free(&t);
}

void or_tmatrix_mblock(double r_ev, double wavelength, double mr, double mi,
                       double axis_ratio, int nmax, int ngauss, int m,
                       double *Tm) {
  struct tables t;
  tables_build(&t, r_ev, wavelength, mr, mi, axis_ratio, nmax, ngauss);
  const int nb = (m == 0) ? nmax : nmax + 1 - m;
  const int n2 = 2 * nb;
  cplx *Q = (cplx *)malloc(sizeof(cplx) * n2 * n2);
  cplx *RgQ = (cplx *)malloc(sizeof(cplx) * n2 * n2);
  assemble(&t, m, Q, RgQ);
  form_t(nb, Q, RgQ, (cplx *)Tm);
  free(Q);
  free(RgQ);
  tables_free(&t);
}

/* T element accessor in the reference index map */
static cplx tel(int nmax, const cplx *T, int i1, int n1, int m, int i2,
                int n2) {
  const cplx *B = T + or_tmatrix_block_offset(nmax, m) / 2;
  if (m > 0) {
    const int nm = nmax + 1 - m;
    return B[(size_t)(i1 * nm + n1 - m) * (2 * nm) + i2 * nm + n2 - m];
  }
  return B[(size_t)(i1 * nmax + n1 - 1) * (2 * nmax) + i2 * nmax + n2 - 1];
}

static void tset(int nmax, cplx *T, int i1, int n1, int m, int i2, int n2,
                 cplx v) {
  cplx *B = T + or_tmatrix_block_offset(nmax, m) / 2;
  if (m > 0) {
    const int nm = nmax + 1 - m;
    B[(size_t)(i1 * nm + n1 - m) * (2 * nm) + i2 * nm + n2 - m] = v;
  } else {
    B[(size_t)(i1 * nmax + n1 - 1) * (2 * nmax) + i2 * nmax + n2 - 1] = v;
  }
}

void or_tmatrix_q(int nmax, const double *Td, double *qsca, double *qext) {
  const cplx *T = (const cplx *)Td;
  double qs = 0.;
  for (int n1 = 1; n1 < nmax + 1; ++n1) {
    for (int n2 = 1; n2 < nmax + 1; ++n2) {
      for (int m1 = 0; m1 < n1 + 1; ++m1) {
        for (int m2 = 0; m2 < n2 + 1; ++m2) {
          if (m1 == m2) {
            const double factor = (m1 > 0) ? 2. : 1.;
            for (int a = 0; a < 2; ++a) {
              for (int b = 0; b < 2; ++b) {
                const cplx v = tel(nmax, T, a, n1, m1, b, n2);
                qs += factor * (creal(v) * creal(v) + cimag(v) * cimag(v));
              }
            }
          }
        }
      }
    }
  }
  double qe = 0.;
  for (int n1 = 1; n1 < nmax + 1; ++n1) {
    for (int m1 = 0; m1 < n1 + 1; ++m1) {
      const double factor = (m1 > 0) ? 2. : 1.;
      for (int a = 0; a < 2; ++a) {
        for (int b = 0; b < 2; ++b) {
          qe += factor * creal(tel(nmax, T, a, n1, m1, b, n1));
        }
      }
    }
  }
  *qsca = qs;
  *qext = qe;
}

int or_tmatrix_converge(double r_ev, double wavelength, double mr, double mi,
                        double axis_ratio, int min_order, int max_order,
                        int glfac, double tolerance, double *T, int *ngauss_out,
                        int *converged_out, double *info) {
  /* TaskManager.hpp:1146-1197 chain + TMatrixM0Task convergence test
   * (TMatrixResource.hpp:758-775) */
  double qsca = 0., qext = 0.;
  double dqs_t = -2., dqe_t = -2.;
  double dqs = -1., dqe = -1.;
  int converged = 0;
  int nmax = 0, ngauss = 0;
  cplx *T0 = (cplx *)malloc(sizeof(cplx) * 4 * (size_t)max_order * max_order);
  for (int order = min_order; order < max_order; ++order) {
    if (converged) {
      break;
    }
    const int ng = glfac * order;
    double nqs, nqe;
    or_tmatrix_m0(r_ev, wavelength, mr, mi, axis_ratio, order, ng,
                  (double *)T0, &nqs, &nqe);
    const double old_qs = qsca, old_qe = qext;
    qsca = nqs;
    qext = nqe;
    nmax = order;
    ngauss = ng;
    if (dqs_t == -2.) {
      dqs_t = -1.;
      dqe_t = -1.;
    } else {
      dqs_t = fabs((old_qs - qsca) / qsca);
      dqe_t = fabs((old_qe - qext) / qext);
    }
    if (dqs_t > 0.) {
      dqs = dqs_t;
      dqe = dqe_t;
      if (dqs_t <= tolerance && dqe_t <= tolerance) {
        converged = 1;
      }
    }
  }
  memcpy(T, T0, sizeof(cplx) * 4 * (size_t)nmax * nmax);
  free(T0);
  for (int m = 1; m <= nmax; ++m) {
    or_tmatrix_mblock(r_ev, wavelength, mr, mi, axis_ratio, nmax, ngauss, m,
                      T + or_tmatrix_block_offset(nmax, m));
  }
  info[0] = qsca;
  info[1] = qext;
  or_tmatrix_q(nmax, T, &info[2], &info[3]);
  info[4] = dqs;
  info[5] = dqe;
  *ngauss_out = ngauss;
  *converged_out = converged;
  return nmax;
}

/* ---------------------------------------------- orientation averaging --- */

/* AlignmentAverageTask::execute, AlignmentAverageTask.hpp:115-215 (Mishchenko
 * 1991 eq. 3.27). The Clebsch-Gordan row depends only on (n1, n2, N), so it
 * is evaluated once per triple here instead of once per m; the values are
 * the same. */
void or_orientation_average(int nmax, const double *Td, const double *coeffs,
                            double *Tad) {
  const cplx *T = (const cplx *)Td;
  cplx *Ta = (cplx *)Tad;
  if (coeffs == NULL) {
    memcpy(Ta, T, sizeof(cplx) * or_tmatrix_size(nmax) / 2);
    return;
  }
  double *cg = (double *)malloc(sizeof(double) * (2 * nmax + 1) * 2);
  const int nblocks = 2 * nmax + 1;
  (void)nblocks;
  for (int n1 = 1; n1 < nmax + 1; ++n1) {
    for (int n2 = 1; n2 < nmax + 1; ++n2) {
      const int n12min = (n1 > n2) ? n1 - n2 : n2 - n1;
      const int n12max = n1 + n2;
      const int M = (n1 < n2) ? n1 : n2;
      /* CG rows for every N */
      double *rows = (double *)malloc(sizeof(double) * (n12max + 1) *
                                      (2 * M + 1));
      for (int N = n12min; N < n12max + 1; ++N) {
        or_clebsch_gordan_row(n1, n2, N, rows + (size_t)N * (2 * M + 1));
      }
      const int mtop = M;
      for (int m = 0; m < mtop + 1; ++m) {
        const int msign = (m % 2 == 0) ? 1 : -1;
        cplx acc[2][2] = {{0., 0.}, {0., 0.}};
        for (int N = n12min; N < n12max + 1; ++N) {
          const double *C = rows + (size_t)N * (2 * M + 1);
          const double pN = coeffs[N];
          for (int m1 = 0; m1 < M + 1; ++m1) {
            const double factor = (m1 == 0) ? 1. : 2.;
            const int m1sign = (m1 % 2 == 0) ? 1 : -1;
            const int mm1sign = m1sign * msign;
            const double CGfac = mm1sign * factor * pN * C[M + m] * C[M + m1];
            if ((N + n12max) % 2 == 0) {
              acc[0][0] += CGfac * tel(nmax, T, 0, n1, m1, 0, n2);
              acc[1][1] += CGfac * tel(nmax, T, 1, n1, m1, 1, n2);
            } else {
              acc[0][1] += CGfac * tel(nmax, T, 0, n1, m1, 1, n2);
              acc[1][0] += CGfac * tel(nmax, T, 1, n1, m1, 0, n2);
            }
          }
        }
        tset(nmax, Ta, 0, n1, m, 0, n2, acc[0][0]);
        tset(nmax, Ta, 0, n1, m, 1, n2, acc[0][1]);
        tset(nmax, Ta, 1, n1, m, 0, n2, acc[1][0]);
        tset(nmax, Ta, 1, n1, m, 1, n2, acc[1][1]);
      }
      free(rows);
    }
  }
  free(cg);
}

/* ----------------------------------------------------------- observables --- */

/* special Wigner tables pi/m = d/sin and tau = d' for one angle:
 * ExtinctionSpecialWignerDResources::execute (ExtinctionCoefficientTask.hpp:
 * 242-415); layout [m][n-1], m = 0..nmax */
struct angle_tab {
  double *dsinx; /* (nmax+1) x nmax */
  double *dd;
};

static void angle_tab_build(struct angle_tab *a, int nmax, double cost,
                            double sint, double sininv) {
  a->dsinx = (double *)calloc((size_t)(nmax + 1) * nmax, sizeof(double));
  a->dd = (double *)calloc((size_t)(nmax + 1) * nmax, sizeof(double));
  for (int m = 0; m <= nmax; ++m) {
    or_wigner_d_sinx(cost, sint, sininv, nmax, m, a->dsinx + (size_t)m * nmax,
                     a->dd + (size_t)m * nmax);
  }
}

static void angle_tab_free(struct angle_tab *a) {
  free(a->dsinx);
  free(a->dd);
}

/* get_forward_scattering_matrix, ExtinctionCoefficientTask.hpp:517-619 (and
 * its copies in AbsorptionCoefficientTask.hpp:612-715 and
 * ScatteringMatrixTask.hpp:588-691): S = (1/k) sum_m sum_nn sum_n c_{nn,n}
 * (pi/tau products) T blocks (2 cos m dphi, 2 sin m dphi) */
static void forward_s(int nmax, const cplx *T, double k,
                      const struct angle_tab *tin, const struct angle_tab *tout,
                      cplx expiphi, cplx *S) {
  S[0] = S[1] = S[2] = S[3] = CX(0., 0.);
  cplx expimphi = CX(1., 0.);
  for (int m = 0; m < nmax + 1; ++m) {
    const int nmin = (m > 1) ? m : 1;
    const double fcos = 2. * creal(expimphi);
    const double fsin = 2. * cimag(expimphi);
    expimphi *= expiphi;
    for (int nn = nmin; nn < nmax + 1; ++nn) {
      const double pi_nn = m * tin->dsinx[(size_t)m * nmax + nn - 1];
      const double tau_nn = tin->dd[(size_t)m * nmax + nn - 1];
      for (int n = nmin; n < nmax + 1; ++n) {
        const double pi_n = m * tout->dsinx[(size_t)m * nmax + n - 1];
        const double tau_n = tout->dd[(size_t)m * nmax + n - 1];
        const cplx c_nnn = cnn(nn, n);
        const cplx T11 = tel(nmax, T, 0, n, m, 0, nn);
        const cplx T22 = tel(nmax, T, 1, n, m, 1, nn);
        if (m == 0) {
          const cplx factor = c_nnn * tau_n * tau_nn;
          S[0] += factor * T22;
          S[3] += factor * T11;
        } else {
          const cplx T12 = tel(nmax, T, 0, n, m, 1, nn);
          const cplx T21 = tel(nmax, T, 1, n, m, 0, nn);
          const cplx real_factor = c_nnn * fcos;
          const cplx imag_factor = c_nnn * fsin;
          const double pi_pi = pi_n * pi_nn;
          const double pi_tau = pi_n * tau_nn;
          const double tau_pi = tau_n * pi_nn;
          const double tau_tau = tau_n * tau_nn;
          S[0] += real_factor * (T11 * pi_pi + T21 * tau_pi + T12 * pi_tau +
                                 T22 * tau_tau);
          S[1] += imag_factor * (T11 * pi_tau + T21 * tau_tau + T12 * pi_pi +
                                 T22 * tau_pi);
          S[2] -= imag_factor * (T11 * tau_pi + T21 * pi_pi + T12 * tau_tau +
                                 T22 * pi_tau);
          S[3] += real_factor * (T11 * tau_tau + T21 * pi_tau + T12 * tau_pi +
                                 T22 * pi_pi);
        }
      }
    }
  }
  const double kinv = 1. / k;
  S[0] *= kinv;
  S[1] *= kinv;
  S[2] *= kinv;
  S[3] *= kinv;
}

static void angle_of(double theta, double *c, double *s, double *si) {
  *c = cos(theta);
  *s = sqrt((1. - *c) * (1. + *c));
  *si = (*s != 0.) ? 1. / *s : 9000.;
}

void or_extinction(int nmax, const double *Td, double wavelength, double r_ev,
                   int ntheta, const double *theta, double *out) {
  const cplx *T = (const cplx *)Td;
  const double k = 2. * M_PI / wavelength;
  for (int it = 0; it < ntheta; ++it) {
    double c, s, si;
    angle_of(theta[it], &c, &s, &si);
    struct angle_tab a;
    angle_tab_build(&a, nmax, c, s, si);
    cplx S[4];
    forward_s(nmax, T, k, &a, &a, CX(1., 0.), S);
    const double prefactor = 2. * M_PI / k;
    double qext = prefactor * cimag(S[0] + S[3]);
    double qpol = prefactor * cimag(S[0] - S[3]);
    double qcpol = prefactor * creal(S[3] - S[0]);
    const double norm = M_PI * r_ev * r_ev;
    out[3 * it + 0] = qext / norm;
    out[3 * it + 1] = qpol / norm;
    out[3 * it + 2] = qcpol / norm;
    angle_tab_free(&a);
  }
}

void or_absorption(int nmax, const double *Td, double wavelength, double r_ev,
                   int ntheta, const double *theta, int ngauss,
                   int account_for_scattering, double *out) {
  /* AbsorptionCoefficientGrid::execute (AbsorptionCoefficientTask.hpp:
   * 211-257) and AbsorptionCoefficientTask::execute (:722-781) */
  const cplx *T = (const cplx *)Td;
  const double k = 2. * M_PI / wavelength;
  struct angle_tab *gin = NULL;
  double *ct = NULL, *wt = NULL, *phi = NULL, *wphi = NULL;
  if (account_for_scattering) {
    ct = (double *)malloc(sizeof(double) * ngauss);
    wt = (double *)malloc(sizeof(double) * ngauss);
    phi = (double *)malloc(sizeof(double) * ngauss);
    wphi = (double *)malloc(sizeof(double) * ngauss);
    or_gauss_legendre(ngauss, ct, wt);
    or_gauss_legendre_ab(ngauss, 0., 2. * M_PI, phi, wphi);
    gin = (struct angle_tab *)malloc(sizeof(struct angle_tab) * ngauss);
    for (int i = 0; i < ngauss; ++i) {
      const double s = sqrt((1. - ct[i]) * (1. + ct[i]));
      const double si = (s != 0.) ? 1. / s : 9000.;
      angle_tab_build(&gin[i], nmax, ct[i], s, si);
    }
  }
  for (int it = 0; it < ntheta; ++it) {
    double c, s, si;
    angle_of(theta[it], &c, &s, &si);
    struct angle_tab a;
    angle_tab_build(&a, nmax, c, s, si);
    cplx S[4];
    forward_s(nmax, T, k, &a, &a, CX(1., -0.), S);
    const double prefactor = 2. * M_PI / k;
    double qabs = prefactor * cimag(S[0] + S[3]);
    double qabspol = prefactor * cimag(S[0] - S[3]);
    if (account_for_scattering) {
      for (int ti = 0; ti < ngauss; ++ti) {
        for (int pi = 0; pi < ngauss; ++pi) {
          cplx St[4];
          forward_s(nmax, T, k, &gin[ti], &a, CX(cos(phi[pi]), -sin(phi[pi])),
                    St);
          const double weight = wt[ti] * wphi[pi];
          const double z00 =
              creal(0.5 * (St[0] * conj(St[0]) + St[1] * conj(St[1]) +
                           St[2] * conj(St[2]) + St[3] * conj(St[3])));
          qabs -= z00 * weight;
          const double z10 =
              creal(0.5 * (St[0] * conj(St[0]) + St[1] * conj(St[1]) -
                           St[2] * conj(St[2]) - St[3] * conj(St[3])));
          qabspol -= z10 * weight;
        }
      }
    }
    const double norm = M_PI * r_ev * r_ev;
    out[2 * it + 0] = qabs / norm;
    out[2 * it + 1] = qabspol / norm;
    angle_tab_free(&a);
  }
  if (account_for_scattering) {
    for (int i = 0; i < ngauss; ++i) {
      angle_tab_free(&gin[i]);
    }
    free(gin);
    free(ct);
    free(wt);
    free(phi);
    free(wphi);
  }
}

void or_scattering_matrix(int nmax, const double *Td, double wavelength,
                          int ntheta, double *out) {
  /* ScatteringMatrixGrid::execute (ScatteringMatrixTask.hpp:207-277) with
   * theta_in = pi/2 (TaskManager.hpp:832-833), ScatteringMatrixTask::execute
   * (:698-751) */
  const cplx *T = (const cplx *)Td;
  const double k = 2. * M_PI / wavelength;
  const int nphi = 2 * ntheta;
  const double cin = cos(M_PI_2);
  const double sin_ = sqrt((1. - cin) * (1. + cin));
  const double sinv = (sin_ != 0.) ? 1. / sin_ : 9000.;
  struct angle_tab ain;
  angle_tab_build(&ain, nmax, cin, sin_, sinv);
  double *ct = (double *)malloc(sizeof(double) * ntheta);
  double *wt = (double *)malloc(sizeof(double) * ntheta);
  double *phi = (double *)malloc(sizeof(double) * nphi);
  double *wphi = (double *)malloc(sizeof(double) * nphi);
  or_gauss_legendre(ntheta, ct, wt);
  or_gauss_legendre_ab(nphi, 0., 2. * M_PI, phi, wphi);
  const cplx I1 = CX(0., 1.);
  for (int it = 0; it < ntheta; ++it) {
    const double s = sqrt((1. - ct[it]) * (1. + ct[it]));
    const double si = (s != 0.) ? 1. / s : 9000.;
    struct angle_tab aout;
    angle_tab_build(&aout, nmax, ct[it], s, si);
    for (int ip = 0; ip < nphi; ++ip) {
      cplx S[4];
      forward_s(nmax, T, k, &ain, &aout, CX(cos(phi[ip]), sin(phi[ip])), S);
      double *Z = out + ((size_t)it * nphi + ip) * 16;
      Z[0] = creal(0.5 * (S[0] * conj(S[0]) + S[1] * conj(S[1]) +
                          S[2] * conj(S[2]) + S[3] * conj(S[3])));
      Z[1] = creal(0.5 * (S[0] * conj(S[0]) - S[1] * conj(S[1]) +
                          S[2] * conj(S[2]) - S[3] * conj(S[3])));
      Z[2] = creal(-S[0] * conj(S[1]) - S[3] * conj(S[2]));
      Z[3] = creal(I1 * (S[0] * conj(S[1]) - S[3] * conj(S[2])));
      Z[4] = creal(0.5 * (S[0] * conj(S[0]) + S[1] * conj(S[1]) -
                          S[2] * conj(S[2]) - S[3] * conj(S[3])));
      Z[5] = creal(0.5 * (S[0] * conj(S[0]) - S[1] * conj(S[1]) -
                          S[2] * conj(S[2]) + S[3] * conj(S[3])));
      Z[6] = creal(-S[0] * conj(S[1]) + S[3] * conj(S[2]));
      Z[7] = creal(I1 * (S[0] * conj(S[1]) + S[3] * conj(S[2])));
      Z[8] = creal(-S[0] * conj(S[2]) - S[3] * conj(S[1]));
      Z[9] = creal(-S[0] * conj(S[2]) + S[3] * conj(S[1]));
      Z[10] = creal(S[0] * conj(S[3]) + S[1] * conj(S[2]));
      Z[11] = creal(-I1 * (S[0] * conj(S[3]) + S[2] * conj(S[1])));
      Z[12] = creal(I1 * (S[2] * conj(S[0]) + S[3] * conj(S[1])));
      Z[13] = creal(I1 * (S[2] * conj(S[0]) - S[3] * conj(S[1])));
      Z[14] = creal(-I1 * (S[3] * conj(S[0]) - S[1] * conj(S[2])));
      Z[15] = creal(S[3] * conj(S[0]) - S[1] * conj(S[2]));
    }
    angle_tab_free(&aout);
  }
  angle_tab_free(&ain);
  free(ct);
  free(wt);
  free(phi);
  free(wphi);
}

/* ------------------------------------------------------------ plain path --- */

/* TMatrixCalculator::calculate_TMatrix (TMatrixCalculator.hpp:64-213): the
 * order loop (ngauss = ndgs nmax) and then the quadrature loop on the m = 0
 * sums. Returns 0, or 1 where the reference aborts ("Unable to converge!"). */
int or_calculator_orders(double r_ev, double wavelength, double mr, double mi,
                         double axis_ratio, int maximum_order, double tolerance,
                         int ndgs, int maximum_ngauss, int *nmax_out,
                         int *ngauss_out) {
  const double xev = 2. * M_PI * r_ev / wavelength;
  int nmax = (int)fmax(4., xev + 4.05 * cbrt(xev));
  double old_qext = 0., old_qsca = 0., dext = 1., dsca = 1.;
  int status = 0;
  while (nmax < maximum_order && (dext > tolerance || dsca > tolerance)) {
    const int ngauss = ndgs * nmax;
    double *T0 = (double *)malloc(sizeof(double) * 8 * nmax * nmax);
    double qsca, qext;
    or_tmatrix_m0(r_ev, wavelength, mr, mi, axis_ratio, nmax, ngauss, T0, &qsca,
                  &qext);
    free(T0);
    dsca = fabs((old_qsca - qsca) / qsca);
    dext = fabs((old_qext - qext) / qext);
    old_qext = qext;
    old_qsca = qsca;
    ++nmax;
  }
  if (nmax == maximum_order) {
    *nmax_out = nmax - 1;
    *ngauss_out = ndgs * (nmax - 1);
    return 1;
  }
  --nmax;
  int ngauss = nmax * ndgs + 1;
  dext = tolerance + 1.;
  dsca = tolerance + 1.;
  while (ngauss < maximum_ngauss && (dext > tolerance || dsca > tolerance)) {
    double *T0 = (double *)malloc(sizeof(double) * 8 * nmax * nmax);
    double qsca, qext;
    or_tmatrix_m0(r_ev, wavelength, mr, mi, axis_ratio, nmax, ngauss, T0, &qsca,
                  &qext);
    free(T0);
    dsca = fabs((old_qsca - qsca) / qsca);
    dext = fabs((old_qext - qext) / qext);
    old_qext = qext;
    old_qsca = qsca;
    ++ngauss;
  }
  if (ngauss == maximum_ngauss) {
    status = 1;
  }
  --ngauss;
  *nmax_out = nmax;
  *ngauss_out = ngauss;
  return status;
}

/* particle-frame direction and amplitude rotation of a lab direction
 * (TMatrix::get_forward_scattering_matrix, TMatrix.hpp:1306-1420) */
struct pdir {
  double c, s, si, cphi, sphi;
  double R[2][2];
};

static void particle_dir(double ca, double sa, double cb, double sb,
                         double theta, double phi, struct pdir *d) {
  const double ct = cos(theta), st = sin(theta);
  const double cp = cos(phi), sp = sin(phi);
  const double cosphirel = cp * ca + sp * sa;
  const double sinphirel = sp * ca - cp * sa;
  const double ctp = ct * cb + st * sb * cosphirel;
  const double stp = sin(acos(ctp));
  if (stp != 0.) {
    d->si = 1. / stp;
    d->cphi = (cb * st * cosphirel - sb * ct) * d->si;
    d->sphi = st * sinphirel * d->si;
  } else {
    d->cphi = 1.;
    d->sphi = 0.;
    d->si = 9000.;
  }
  d->c = ctp;
  d->s = stp;
  const double B[3][3] = {{ca * cb, sa * cb, -sb}, {-sa, ca, 0.}, {ca * sb, sa * sb, cb}};
  const double AL[3][2] = {{ct * cp, -sp}, {ct * sp, cp}, {-st, 0.}};
  const double AP[2][3] = {{ctp * d->cphi, ctp * d->sphi, -stp}, {-d->sphi, d->cphi, 0.}};
  double C[3][2];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 2; ++j) {
      C[i][j] = 0.;
      for (int k = 0; k < 3; ++k) {
        C[i][j] += B[i][k] * AL[k][j];
      }
    }
  }
  for (int i = 0; i < 2; ++i) {
    for (int j = 0; j < 2; ++j) {
      d->R[i][j] = 0.;
      for (int k = 0; k < 3; ++k) {
        d->R[i][j] += AP[i][k] * C[k][j];
      }
    }
  }
}

void or_amplitude_lab(int nmax, const double *Td, double wavelength, double alpha,
                      double beta, double theta_in, double phi_in,
                      double theta_out, double phi_out, double *Sout) {
  const cplx *T = (const cplx *)Td;
  const double k = 2. * M_PI / wavelength;
  const double ca = cos(alpha), sa = sin(alpha), cb = cos(beta), sb = sin(beta);
  struct pdir din, dout;
  particle_dir(ca, sa, cb, sb, theta_in, phi_in, &din);
  particle_dir(ca, sa, cb, sb, theta_out, phi_out, &dout);
  struct angle_tab ain, aout;
  angle_tab_build(&ain, nmax, din.c, din.s, din.si);
  angle_tab_build(&aout, nmax, dout.c, dout.s, dout.si);
  const cplx e1 = CX(dout.cphi * din.cphi + dout.sphi * din.sphi,
                     dout.sphi * din.cphi - dout.cphi * din.sphi);
  cplx S[4];
  forward_s(nmax, T, k, &ain, &aout, e1, S);
  angle_tab_free(&ain);
  angle_tab_free(&aout);
  /* S^L = R_out^-1 S^P R_in (TMatrix.hpp:1420-1460) */
  double Ro[2][2];
  const double det = 1. / (dout.R[0][0] * dout.R[1][1] - dout.R[0][1] * dout.R[1][0]);
  Ro[0][0] = dout.R[1][1] * det;
  Ro[0][1] = -dout.R[0][1] * det;
  Ro[1][0] = -dout.R[1][0] * det;
  Ro[1][1] = dout.R[0][0] * det;
  const cplx cS11 = S[0] * din.R[0][0] + S[1] * din.R[1][0];
  const cplx cS12 = S[0] * din.R[0][1] + S[1] * din.R[1][1];
  const cplx cS21 = S[2] * din.R[0][0] + S[3] * din.R[1][0];
  const cplx cS22 = S[2] * din.R[0][1] + S[3] * din.R[1][1];
  const cplx L[4] = {Ro[0][0] * cS11 + Ro[0][1] * cS21, Ro[0][0] * cS12 + Ro[0][1] * cS22,
                     Ro[1][0] * cS11 + Ro[1][1] * cS21, Ro[1][0] * cS12 + Ro[1][1] * cS22};
  for (int q = 0; q < 4; ++q) {
    Sout[2 * q] = creal(L[q]);
    Sout[2 * q + 1] = cimag(L[q]);
  }
}

/* Z (TMatrix.hpp:1896-1948) and K (:1972-2010) from S, row major */
void or_z_from_s(const double *Sd, double *Z) {
  const cplx *S = (const cplx *)Sd;
  const cplx I1 = CX(0., 1.);
  Z[0] = creal(0.5 * (S[0] * conj(S[0]) + S[1] * conj(S[1]) + S[2] * conj(S[2]) +
                      S[3] * conj(S[3])));
  Z[1] = creal(0.5 * (S[0] * conj(S[0]) - S[1] * conj(S[1]) + S[2] * conj(S[2]) -
                      S[3] * conj(S[3])));
  Z[2] = creal(-S[0] * conj(S[1]) - S[3] * conj(S[2]));
  Z[3] = creal(I1 * (S[0] * conj(S[1]) - S[3] * conj(S[2])));
  Z[4] = creal(0.5 * (S[0] * conj(S[0]) + S[1] * conj(S[1]) - S[2] * conj(S[2]) -
                      S[3] * conj(S[3])));
  Z[5] = creal(0.5 * (S[0] * conj(S[0]) - S[1] * conj(S[1]) - S[2] * conj(S[2]) +
                      S[3] * conj(S[3])));
  Z[6] = creal(-S[0] * conj(S[1]) + S[3] * conj(S[2]));
  Z[7] = creal(I1 * (S[0] * conj(S[1]) + S[3] * conj(S[2])));
  Z[8] = creal(-S[0] * conj(S[2]) - S[3] * conj(S[1]));
  Z[9] = creal(-S[0] * conj(S[2]) + S[3] * conj(S[1]));
  Z[10] = creal(S[0] * conj(S[3]) + S[1] * conj(S[2]));
  Z[11] = creal(-I1 * (S[0] * conj(S[3]) + S[2] * conj(S[1])));
  Z[12] = creal(I1 * (S[2] * conj(S[0]) + S[3] * conj(S[1])));
  Z[13] = creal(I1 * (S[2] * conj(S[0]) - S[3] * conj(S[1])));
  Z[14] = creal(-I1 * (S[3] * conj(S[0]) - S[1] * conj(S[2])));
  Z[15] = creal(S[3] * conj(S[0]) - S[1] * conj(S[2]));
}

void or_k_from_s(double wavelength, const double *Sd, double *K) {
  const cplx *S = (const cplx *)Sd;
  const double pf = 2. * M_PI / (2. * M_PI / wavelength);
  for (int i = 0; i < 16; ++i) {
    K[i] = 0.;
  }
  K[0] = pf * cimag(S[0] + S[3]);
  K[5] = K[10] = K[15] = K[0];
  K[1] = K[4] = pf * cimag(S[0] - S[3]);
  K[2] = K[8] = -pf * cimag(S[1] + S[2]);
  K[3] = K[12] = pf * creal(S[2] - S[1]);
  K[6] = pf * cimag(S[2] - S[1]);
  K[9] = -K[6];
  K[7] = -pf * creal(S[1] + S[2]);
  K[13] = -K[7];
  K[11] = pf * creal(S[3] - S[0]);
  K[14] = -K[11];
}
