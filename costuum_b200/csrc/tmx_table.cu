// Host side of the orientation/shape-averaged observables: orientation
// distribution coefficients, shape distribution nodes, and the get_table
// pipeline (T-matrices -> orientation average -> S -> Q / Z -> shape average).
//
// Reference (CosTuuM): CTMModule.cpp:146-478 (get_table), TaskManager.hpp:
// 445-1346 (the per-grain task graph), OrientationDistribution.hpp:220-243,
// MishchenkoOrientationDistribution.hpp:107-118,
// DavisGreensteinOrientationDistribution.hpp:81-102,
// ShapeDistribution.hpp:95-106, DraineHensleyShapeDistribution.hpp.
#include <cmath>
#include <complex>
#include <cstring>
#include <system_error>
#include <thread>
#include <vector>

#include "tmx_ctx.h"

// ------------------------------------------------------ quadrature tools --

// Gauss-Legendre rule on [a, b] (get_gauss_legendre_points_and_weights_ab,
// SpecialFunctions.hpp:737-751)
static void gl_ab(int order, double a, double b, double *x, double *w) {
  tmx_host_gauss_legendre(order, x, w);
  const double wfac = 0.5 * (b - a);
  const double xterm = 0.5 * (a + b);
  for (int i = 0; i < order; ++i) {
    x[i] = wfac * x[i] + xterm;
    w[i] *= wfac;
  }
}

// Adaptive Gauss-Legendre quadrature that raises the order by one until
// either the absolute or the relative change is below its target
// (gauss_legendre_quadrature, SpecialFunctions.hpp:771-810).
template <typename F>
static double gl_quadrature(F f, double lower, double upper, int start,
                            int maximum, double abs_tol, double rel_tol) {
  int order = start;
  double old_q = 0.;
  double absd = abs_tol + 1.;
  double reld = rel_tol + 1.;
  std::vector<double> x(maximum > 0 ? maximum : 1), w(x.size());
  while (order < maximum && absd > abs_tol && reld > rel_tol) {
    gl_ab(order, lower, upper, x.data(), w.data());
    double q = 0.;
    for (int i = 0; i < order; ++i) {
      q += w[i] * f(x[i]);
    }
    absd = fabs(q - old_q);
    reld = absd / fabs(q + old_q);
    old_q = q;
    ++order;
  }
  return old_q;
}

// Legendre P_n(cos beta) = d^n_00(beta) by the m = 0 recurrence of
// SpecialFunctions::wigner_dn_0m (SpecialFunctions.hpp:302-371)
static double wigner_d00(double cosx, int order) {
  if (order == 0) {
    return 1.;
  }
  double d1 = 1., d2 = cosx, last = cosx;
  for (int n = 0; n < order; ++n) {
    const double np1 = n + 1.;
    const double np2 = n + 2.;
    const double np12p1 = 2. * np1 + 1.;
    const double dnp1 = (np12p1 * cosx * d2 - np1 * d1) / np2;
    last = d2;
    d1 = d2;
    d2 = dnp1;
  }
  return last;
}

// ------------------------------------------------------- distributions ---

extern "C" int tmx_orientation_coefficients(int kind, double param, int order,
                                            double (*fn)(double, void *),
                                            void *arg, double *out) {
  if (order < 0 || !out || kind < 0 || kind > 3 || (kind == 3 && !fn)) {
    return TMX_ERR_INVALID;
  }
  for (int i = 0; i <= order; ++i) {
    out[i] = 0.;
  }
  if (kind == 1) {
    // Mishchenko: p(beta) = 1/2 + 5/4 p2 (3 cos^2 - 1), p2 = 3/2 <cos^2> - 1/2
    out[0] = 1.;
    if (order >= 2) {
      out[2] = 1.5 * param - 0.5;
    }
    return TMX_OK;
  }
  if (kind == 2) {
    // Davis-Greenstein perfect alignment
    if (param < 1.) {
      double nominator = 1., denominator = 2.;
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
    return TMX_OK;
  }
  // numerical: random (p = 1/2; tolerances 1e-10 / 1e-5) or custom
  // (Python function; tolerances 1e-4 / 1e-4, PyOrientationDistribution.hpp)
  auto p = [&](double beta) { return kind == 0 ? 0.5 : fn(beta, arg); };
  const double at = (kind == 0) ? 1.e-10 : 1.e-4;
  const double rt = (kind == 0) ? 1.e-5 : 1.e-4;
  const double norm = gl_quadrature(
      [&](double beta) { return sin(beta) * p(beta); }, 0., M_PI, 100, 1000,
      at, rt);
  const double nf = 1. / norm;
  out[0] = 1.;
  auto coefficient = [&](int i) {
    return gl_quadrature(
        [&](double beta) {
          const double cb = cos(beta);
          const double sb = sin(beta);
          const double pb = nf * p(beta);
          return sb * pb * wigner_d00(cb, i);
        },
        0., M_PI, 2 * (i + 1), 100 * (i + 1), at, rt);
  };
  // the coefficients are independent quadratures (their cost grows with
  // the order): random orientation spreads them over host threads,
  // interleaved; a custom p(beta) calls into Python and stays on this thread
  if (kind == 0 && order >= 32) {
    const int nt = std::max(
        1, std::min<int>((int)std::thread::hardware_concurrency(), 32));
    std::vector<std::thread> pool;
    int started = 0;
    try {
      for (int t = 0; t < nt; ++t) {
        pool.emplace_back([&, t]() {
          for (int i = 1 + t; i <= order; i += nt) {
            out[i] = coefficient(i);
          }
        });
        ++started;
      }
    } catch (const std::system_error &) {
      // fewer threads than asked for: the residues of the missing ones below
    }
    for (std::thread &th : pool) {
      th.join();
    }
    for (int t = started; t < nt; ++t) {
      for (int i = 1 + t; i <= order; i += nt) {
        out[i] = coefficient(i);
      }
    }
    return TMX_OK;
  }
  for (int i = 1; i <= order; ++i) {
    out[i] = coefficient(i);
  }
  return TMX_OK;
}

namespace {

// DraineHensleyShapeDistribution helpers (DraineHensleyShapeDistribution.hpp)
double dh_shape_factor(double d) {
  if (d < 1.) {
    const double e2 = 1. - d * d;
    const double e = sqrt(e2);
    return (1. - e2) * (0.5 * log((1. + e) / (1. - e)) / e - 1.) / e2;
  } else if (d > 1.) {
    const double e2 = 1. - 1. / (d * d);
    const double e = sqrt(e2);
    return (1. - sqrt(1. - e2) * asin(e) / e) / e2;
  }
  return 1. / 3.;
}

double dh_jacobian(double d) {
  if (d < 1.) {
    const double e2 = 1. - d * d;
    if (e2 < 1.e-5) {
      return 4. / 15. + 2. * e2 / 21. + 3. * e2 * e2 / 70.;
    }
    const double e = sqrt(e2);
    return 0.5 * sqrt(1. - e2) * ((3. - e2) * log((1. + e) / (1. - e)) - 6. * e) /
           (e2 * e2 * e);
  } else if (d > 1.) {
    const double e2 = 1. - 1. / (d * d);
    if (e2 < 1.e-5) {
      return 4. / 15. - 2. * e2 / 21. - 11. * e2 * e2 / 210.;
    }
    const double e = sqrt(e2);
    return (1. - e2) * ((3. - 2. * e2) * asin(e) - 3. * e * sqrt(1. - e2)) /
           (e2 * e2 * e);
  }
  return 4. / 15.;
}

double dh_cde2(double L) {
  const double Lm1 = L - 1.;
  return 12. * L * Lm1 * Lm1;
}

double dh_eval(double d) { return dh_cde2(dh_shape_factor(d)) * dh_jacobian(d); }

} // namespace

// kind 0: the default ShapeDistribution (exp(-(d-1)^2 / (2 x 0.027777778))
// on [0.5, 1.5]); kind 1: Draine & Hensley (2017) CDE2 with a probability
// cutoff (param1) or a prolate/oblate fraction (param2 > 0)
extern "C" int tmx_shape_distribution(int kind, int npoints, double param1,
                                      double param2, double *shapes,
                                      double *weights, double *limits) {
  if (npoints < 1 || !shapes || !weights || kind < 0 || kind > 1) {
    return TMX_ERR_INVALID;
  }
  double dmin = 0.5, dmax = 1.5;
  auto pdf = [&](double d) -> double {
    if (kind == 0) {
      if (d >= 0.5 && d <= 1.5) {
        const double x = d - 1.;
        return exp(-0.5 * x * x / 0.027777778);
      }
      return 0.;
    }
    return (d >= dmin && d <= dmax) ? dh_eval(d) : 0.;
  };
  if (kind == 1) {
    const double cutoff = param1, fraction = param2;
    if (fraction > 0.) {
      auto integ = [&](double a, double b) {
        return gl_quadrature([&](double d) { return dh_eval(d); }, a, b, 10,
                             1000, 1.e-10, 1.e-10);
      };
      const double prolate_fraction = integ(0., 1.);
      const double prolate_target = fraction * prolate_fraction;
      double lower = 0., upper = 1., half = 0.5;
      double integral = integ(half, 1.);
      int guard = 0;
      while (fabs(integral - prolate_target) >
                 0.005 * fabs(integral + prolate_target) &&
             ++guard < 200) {
        if (integral > prolate_target) {
          lower = half;
        } else {
          upper = half;
        }
        half = 0.5 * (lower + upper);
        integral = integ(half, 1.);
      }
      dmin = half;
      const double oblate_target = fraction * (1. - prolate_fraction);
      lower = 1.;
      upper = 2.;
      integral = integ(1., upper);
      guard = 0;
      while (integral < oblate_target && ++guard < 60) {
        upper *= 2.;
        integral = integ(1., upper);
      }
      half = 0.5 * (lower + upper);
      integral = integ(1., half);
      guard = 0;
      while (fabs(integral - oblate_target) > 1.e-5 * fabs(integral + oblate_target) &&
             ++guard < 200) {
        if (integral > oblate_target) {
          upper = half;
        } else {
          lower = half;
        }
        half = 0.5 * (lower + upper);
        integral = integ(1., half);
      }
      dmax = half;
    } else {
      dmin = 1.;
      dmax = 1.;
      double valmin = pdf(dmin) - cutoff;
      int guard = 0;
      while (valmin > 0. && ++guard < 200) {
        dmin *= 0.5;
        valmin = pdf(dmin) - cutoff;
      }
      double ub = 1.;
      guard = 0;
      while (fabs(dmin - ub) > 0.005 * fabs(dmin + ub) && ++guard < 200) {
        const double mid = 0.5 * (dmin + ub);
        const double v = pdf(mid) - cutoff;
        if (v < 0.) {
          dmin = mid;
        } else {
          ub = mid;
        }
      }
      double valmax = pdf(dmax) - cutoff;
      guard = 0;
      while (valmax > 0. && ++guard < 1000) {
        dmax += 1.;
        valmax = pdf(dmax) - cutoff;
      }
      double lb = 1.;
      guard = 0;
      while (fabs(dmax - lb) > 0.005 * fabs(dmax + lb) && ++guard < 200) {
        const double mid = 0.5 * (lb + dmax);
        const double v = pdf(mid) - cutoff;
        if (v > 0.) {
          lb = mid;
        } else {
          dmax = mid;
        }
      }
    }
  }
  if (limits) {
    limits[0] = dmin;
    limits[1] = dmax;
  }
  // ShapeDistribution::evaluate: GL nodes on [dmin, dmax], weight x p(d)
  gl_ab(npoints, dmin, dmax, shapes, weights);
  for (int i = 0; i < npoints; ++i) {
    weights[i] *= pdf(shapes[i]);
  }
  return TMX_OK;
}

// R_V / R_S of a spheroid (get_equal_volume_to_equal_surface_area_sphere_
// ratio, SpecialFunctions.hpp:557-583)
extern "C" double tmx_rv_over_rs(double d) {
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

// -------------------------------------------------------------- get_table --

namespace {

// zenith angle as the reference's grids compute it
TmxAngle make_angle(double cost) {
  TmxAngle a;
  a.c = cost;
  a.s = sqrt((1. - cost) * (1. + cost));
  a.si = (a.s != 0.) ? 1. / a.s : 9000.;
  return a;
}

int64_t est_nmax(double x, int min_order, int max_order) {
  double e = x + 4.05 * cbrt(x) + 8.;
  e = std::max<double>(e, min_order);
  return std::min<int64_t>((int64_t)e, max_order - 1);
}

// Work plan of the observable kernels for the grains `og` (already on the
// device in ctx->o_og) and the amplitude jobs `sj` (already in ctx->o_sj):
// the first (n1, n2) pair of every grain for the orientation kernel and
// groups of at most 32 consecutive jobs of one grain for the amplitude
// kernel.
int upload_obs_plan(tmx_ctx *ctx, const std::vector<TmxObsGrain> &og,
                    const std::vector<TmxSJob> &sj) {
  int rc0;
  ++ctx->plan_seq;
  cudaStream_t st = ctx->stream;
  const int64_t n = (int64_t)og.size();
  // orientation-average work items, pair-major (tmx_launch_orient_pairs):
  // grains by descending order; pair (n1, n2) has one item per grain of
  // order >= max(n1, n2)
  int nbmax = 1;
  for (int64_t g = 0; g < n; ++g) {
    nbmax = std::max(nbmax, og[g].nmax);
  }
  std::vector<int32_t> order;
  for (int64_t g = 0; g < n; ++g) {
    if (og[g].nmax > 0) {
      order.push_back((int32_t)g);
    }
  }
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    return og[a].nmax > og[b].nmax;
  });
  std::vector<int64_t> at_least(nbmax + 2, 0); // grains of order >= k
  for (int32_t g : order) {
    at_least[og[g].nmax] += 1;
  }
  for (int k = nbmax; k >= 1; --k) {
    at_least[k] += at_least[k + 1];
  }
  std::vector<int64_t> base((size_t)nbmax * nbmax + 1, 0);
  int64_t npairs = 0;
  for (int n1 = 1; n1 <= nbmax; ++n1) {
    for (int n2 = 1; n2 <= nbmax; ++n2) {
      base[(size_t)(n1 - 1) * nbmax + (n2 - 1)] = npairs;
      npairs += at_least[std::max(n1, n2)];
    }
  }
  base.back() = npairs;
  if ((rc0 = ensure(ctx, ctx->o_ord, std::max<size_t>(1, order.size()) * sizeof(int32_t)))) {
    return rc0;
  }
  if (!order.empty()) {
    CK(cudaMemcpyAsync(ctx->o_ord.p, order.data(), order.size() * sizeof(int32_t),
                       cudaMemcpyHostToDevice, st));
  }
  std::vector<TmxAmpGroup> grp;
  for (size_t j = 0; j < sj.size(); ++j) {
    if (grp.empty() || grp.back().grain != sj[j].grain || grp.back().njobs == 32) {
      TmxAmpGroup a;
      a.grain = sj[j].grain;
      a.njobs = 0;
      a.job0 = (int64_t)j;
      grp.push_back(a);
    }
    grp.back().njobs += 1;
  }
  int rc;
  if ((rc = ensure(ctx, ctx->o_pairs, base.size() * sizeof(int64_t))) ||
      (rc = ensure(ctx, ctx->o_grp, std::max<size_t>(1, grp.size()) * sizeof(TmxAmpGroup)))) {
    return rc;
  }
  CK(cudaMemcpyAsync(ctx->o_pairs.p, base.data(), base.size() * sizeof(int64_t),
                     cudaMemcpyHostToDevice, st));
  if (!grp.empty()) {
    CK(cudaMemcpyAsync(ctx->o_grp.p, grp.data(), grp.size() * sizeof(TmxAmpGroup),
                       cudaMemcpyHostToDevice, st));
  }
  CK(cudaStreamSynchronize(st));
  ctx->o_ngrains = n;
  ctx->o_npairs = npairs;
  ctx->o_nbmax = nbmax;
  ctx->o_pmax = nbmax;
  ctx->o_ngrp = (int)grp.size();
  if (ctx->profiling) {
    // flops of one matrix set over the kernels' index spaces: the
    // orientation average 16 (2M + 1)(M + 1) per (n1, n2), M = min(n1, n2),
    // of every averaged grain; the amplitudes 16 (2 nb)^2 per m block and job
    double fo = 0., fa = 0.;
    std::vector<double> per_job(nbmax + 1, -1.);
    for (int64_t g = 0; g < n; ++g) {
      const int N = og[g].nmax;
      if (N > 0 && og[g].coef_set >= 0) {
        for (int a = 1; a <= N; ++a) {
          for (int b = 1; b <= N; ++b) {
            const double M = std::min(a, b);
            fo += 16. * (2. * M + 1.) * (M + 1.);
          }
        }
      }
    }
    for (const TmxSJob &j : sj) {
      const int N = og[j.grain].nmax;
      if (N <= 0) {
        continue;
      }
      if (per_job[N] < 0.) {
        double s = 16. * 4. * N * N;
        for (int k = 1; k <= N; ++k) {
          s += 16. * 4. * k * k;
        }
        per_job[N] = s;
      }
      fa += per_job[N];
    }
    ctx->o_fl_orient = fo;
    ctx->o_fl_amp = fa;
  }
  return TMX_OK;
}

// Ta = orientation average (or copy) of Tsrc with the amplitude factors
// folded in, then the amplitudes S of every job (zeroed first: grains with
// nmax 0 have no jobs)
int run_amplitudes(tmx_ctx *ctx, const cplx *const *Tsrc, int nmat,
                   int64_t t_total, int ncoef, cplx *const *S_out,
                   int64_t s_total) {
  cudaStream_t st = ctx->stream;
  int rc;
  if ((rc = ensure(ctx, ctx->Ta,
                   std::max<int64_t>(1, nmat * t_total) * sizeof(cplx)))) {
    return rc;
  }
  for (int k = 0; k < nmat; ++k) {
    CK(cudaMemsetAsync(S_out[k], 0, std::max<int64_t>(0, s_total) * 4 * sizeof(cplx),
                       st));
  }
  if (t_total <= 0 || ctx->o_npairs <= 0) {
    return TMX_OK;
  }
  TmxMatSet avg = {}, amp = {};
  for (int k = 0; k < nmat; ++k) {
    avg.src[k] = Tsrc[k];
    avg.dst[k] = (cplx *)ctx->Ta.p + k * t_total;
    amp.src[k] = avg.dst[k];
    amp.dst[k] = S_out[k];
  }
  const int grid = tmx_amp_grid(ctx->o_nbmax, nmat);
  if ((rc = ensure(ctx, ctx->o_x,
                   (size_t)grid * nmat * 32 * (ctx->o_nbmax + 1) * 4 * sizeof(cplx)))) {
    return rc;
  }
  cudaEvent_t pe = nullptr;
  if ((rc = prof_begin(ctx, TMX_PROF_ORIENT, &pe))) {
    return rc;
  }
  tmx_launch_orient_pairs((const TmxObsGrain *)ctx->o_og.p,
                          (const int64_t *)ctx->o_pairs.p, (const int32_t *)ctx->o_ord.p,
                          ctx->o_pmax, ctx->o_npairs, avg, nmat,
                          (const double *)ctx->o_coef.p,
                          ncoef, (const int64_t *)ctx->cg_off.p,
                          (const double *)ctx->cg.p, ctx->cg_nmax, ctx->o_nbmax, 1,
                          st);
  LAUNCHED();
  // T-matrices in and averaged T-matrices out, once each
  if ((rc = prof_end(ctx, TMX_PROF_ORIENT, pe, nmat * ctx->o_fl_orient, st,
                     2. * nmat * t_total * sizeof(cplx)))) {
    return rc;
  }
  if ((rc = prof_begin(ctx, TMX_PROF_AMP, &pe))) {
    return rc;
  }
  // the pi / tau columns of every angle of the plan, once for all grains
  // (unless the table would be large: then each CTA runs the recurrences)
  const double *wpi = nullptr, *wtau = nullptr;
  const int wn = ctx->o_nbmax;
  const size_t wcol = (size_t)ctx->o_nangles * (wn + 1) * wn;
  if (ctx->o_nangles > 0 && 2 * wcol * sizeof(double) <= ((size_t)512 << 20)) {
    if ((rc = ensure(ctx, ctx->o_wcol, 2 * wcol * sizeof(double)))) {
      return rc;
    }
    wpi = (const double *)ctx->o_wcol.p;
    wtau = wpi + wcol;
    tmx_launch_wigner_cols((const TmxAngle *)ctx->o_angles.p, ctx->o_nangles, wn,
                           (double *)ctx->o_wcol.p, (double *)ctx->o_wcol.p + wcol, st);
    LAUNCHED();
  }
  tmx_launch_amp((const TmxAmpGroup *)ctx->o_grp.p, ctx->o_ngrp,
                 (const TmxSJob *)ctx->o_sj.p, (const TmxObsGrain *)ctx->o_og.p, amp,
                 nmat, (const TmxAngle *)ctx->o_angles.p, (const cplx *)ctx->o_phis.p,
                 (cplx *)ctx->o_x.p, ctx->o_nbmax, grid, wpi, wtau, wn, st);
  LAUNCHED();
  // averaged T-matrices in, four complex amplitudes per job and azimuth out
  if ((rc = prof_end(ctx, TMX_PROF_AMP, pe, nmat * ctx->o_fl_amp, st,
                     nmat * (t_total + 4. * s_total) * sizeof(cplx)))) {
    return rc;
  }
  return TMX_OK;
}

int run_amplitudes(tmx_ctx *ctx, const cplx *Tsrc, int64_t t_total, int ncoef,
                   cplx *S_out, int64_t s_total) {
  return run_amplitudes(ctx, &Tsrc, 1, t_total, ncoef, &S_out, s_total);
}

} // namespace

extern "C" int tmx_get_table(
    tmx_ctx *ctx, int32_t ntypes, int32_t nsizes, const double *sizes,
    int32_t nlambda, const double *lambdas, int32_t ntheta,
    const double *thetas, int32_t nshape, const double *shapes,
    const double *shape_weights, const double *mr, const double *mi,
    const int32_t *orient_set, int32_t nsets, const double *coeffs,
    int32_t ncoef, int32_t flags, int32_t ngauss, const tmx_schedule *sched,
    double *out_q, double *out_z, int32_t *grain_status) {
  if (!ctx) {
    return TMX_ERR_INVALID;
  }
  const bool do_abs = flags & TMX_TABLE_ABSORPTION;
  const bool do_ext = flags & TMX_TABLE_EXTINCTION;
  const bool do_sca = flags & TMX_TABLE_SCATTERING;
  const bool account = (flags & TMX_TABLE_ACCOUNT_FOR_SCATTERING) && do_abs;
  if (ntypes < 0 || nsizes < 0 || nlambda < 0 || ntheta < 0 || nshape < 1 ||
      !sizes || !lambdas || (ntheta > 0 && !thetas) || !shapes ||
      !shape_weights || !mr || !mi || !orient_set || nsets < 0 ||
      (nsets > 0 && (!coeffs || ncoef < 1)) || (account && ngauss < 1) ||
      ((do_abs || do_ext) && !out_q) || (do_sca && !out_z)) {
    return fail(ctx, TMX_ERR_INVALID, "tmx_get_table: invalid arguments");
  }
  tmx_schedule S = {10, 100, 2, 0, 1.e-4};
  if (sched) {
    S = *sched;
  }
  for (int i = 0; i < nsizes * nshape; ++i) {
    if (orient_set[i] >= nsets) {
      return fail(ctx, TMX_ERR_INVALID, "tmx_get_table: orientation set index");
    }
  }
  const int nq = (do_abs ? 2 : 0) + (do_ext ? 3 : 0);
  const int nphi_sca = 2 * ntheta;
  const int64_t ncells = (int64_t)ntypes * nsizes * nlambda;
  if (ncells == 0 || ntheta == 0 || (!do_abs && !do_ext && !do_sca)) {
    return TMX_OK;
  }
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  int rc;
  NvtxRange range("tmx_get_table");

  // ---- angle and azimuth tables
  std::vector<TmxAngle> ang;
  for (int i = 0; i < ntheta; ++i) {
    ang.push_back(make_angle(cos(thetas[i])));
  }
  const int acc_a0 = (int)ang.size();
  std::vector<double> acc_w; // [theta weights (ngauss), phi weights (ngauss)]
  std::vector<cplx> phis;
  phis.push_back(mkc(1., 0.)); // azimuth 0 for the theta -> theta amplitude
  int64_t acc_p0 = 0, sca_p0 = 0;
  if (account) {
    std::vector<double> ct(ngauss), wt(ngauss), ph(ngauss), wp(ngauss);
    tmx_host_gauss_legendre(ngauss, ct.data(), wt.data());
    gl_ab(ngauss, 0., 2. * M_PI, ph.data(), wp.data());
    for (int i = 0; i < ngauss; ++i) {
      ang.push_back(make_angle(ct[i]));
    }
    acc_w = wt;
    acc_w.insert(acc_w.end(), wp.begin(), wp.end());
    acc_p0 = (int64_t)phis.size();
    for (int i = 0; i < ngauss; ++i) {
      phis.push_back(mkc(cos(ph[i]), -sin(ph[i])));
    }
  }
  int sca_ain = -1, sca_a0 = -1;
  if (do_sca) {
    sca_ain = (int)ang.size();
    ang.push_back(make_angle(cos(M_PI_2)));
    sca_a0 = (int)ang.size();
    std::vector<double> ct(ntheta), wt(ntheta), ph(nphi_sca), wp(nphi_sca);
    tmx_host_gauss_legendre(ntheta, ct.data(), wt.data());
    for (int i = 0; i < ntheta; ++i) {
      // theta_out = acos(GL node); the grid keeps cos(theta_out) = node
      ang.push_back(make_angle(ct[i]));
    }
    gl_ab(nphi_sca, 0., 2. * M_PI, ph.data(), wp.data());
    sca_p0 = (int64_t)phis.size();
    for (int i = 0; i < nphi_sca; ++i) {
      phis.push_back(mkc(cos(ph[i]), sin(ph[i])));
    }
  }
  if ((rc = ensure(ctx, ctx->o_angles, ang.size() * sizeof(TmxAngle))) ||
      (rc = ensure(ctx, ctx->o_phis, phis.size() * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->o_wts, std::max<size_t>(1, acc_w.size()) * sizeof(double))) ||
      (rc = ensure(ctx, ctx->o_coef, std::max<int64_t>(1, (int64_t)nsets * ncoef) * sizeof(double))) ||
      (rc = ensure(ctx, ctx->o_shw, nshape * sizeof(double)))) {
    return rc;
  }
  ++ctx->plan_seq; // the observable buffers change below
  CK(cudaMemcpyAsync(ctx->o_angles.p, ang.data(), ang.size() * sizeof(TmxAngle),
                     cudaMemcpyHostToDevice, st));
  ctx->o_nangles = (int)ang.size();
  CK(cudaMemcpyAsync(ctx->o_phis.p, phis.data(), phis.size() * sizeof(cplx),
                     cudaMemcpyHostToDevice, st));
  if (!acc_w.empty()) {
    CK(cudaMemcpyAsync(ctx->o_wts.p, acc_w.data(), acc_w.size() * sizeof(double),
                       cudaMemcpyHostToDevice, st));
  }
  if (nsets > 0) {
    CK(cudaMemcpyAsync(ctx->o_coef.p, coeffs, (int64_t)nsets * ncoef * sizeof(double),
                       cudaMemcpyHostToDevice, st));
  }
  CK(cudaMemcpyAsync(ctx->o_shw.p, shape_weights, nshape * sizeof(double),
                     cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st)); // host vectors above are about to change

  // ---- chunks of whole cells (all shapes of a cell stay together)
  const int64_t per_grain_s =
      ntheta + (account ? (int64_t)ntheta * ngauss * ngauss : 0) +
      (do_sca ? (int64_t)ntheta * nphi_sca : 0);
  const double budget = 6.e9; // bytes for T, Ta and S of one chunk
  std::vector<double> gr_r, gr_l, gr_mr, gr_mi, gr_d;
  int64_t c0 = 0;
  while (c0 < ncells) {
    // grow the chunk until the estimated memory reaches the budget
    int64_t c1 = c0;
    double bytes = 0.;
    while (c1 < ncells) {
      const int64_t isz = (c1 / nlambda) % nsizes;
      const int64_t il = c1 % nlambda;
      double cell = 0.;
      for (int s = 0; s < nshape; ++s) {
        const double x = 2. * M_PI * sizes[isz] / lambdas[il] * std::max(1., cbrt(shapes[s]));
        const int64_t N = est_nmax(x, S.min_order, S.max_order);
        cell += 2. * tmx_tmatrix_size((int32_t)N) * 16. + per_grain_s * 64.;
      }
      if (c1 > c0 && bytes + cell > budget) {
        break;
      }
      bytes += cell;
      ++c1;
      if ((c1 - c0) * nshape >= 32768) {
        break;
      }
    }
    const int64_t nc = c1 - c0;
    const int64_t ng = nc * nshape;
    gr_r.resize(ng);
    gr_l.resize(ng);
    gr_mr.resize(ng);
    gr_mi.resize(ng);
    gr_d.resize(ng);
    for (int64_t c = 0; c < nc; ++c) {
      const int64_t cell = c0 + c;
      const int64_t isz = (cell / nlambda) % nsizes;
      const int64_t il = cell % nlambda;
      for (int s = 0; s < nshape; ++s) {
        const int64_t g = c * nshape + s;
        gr_r[g] = sizes[isz];
        gr_l[g] = lambdas[il];
        gr_mr[g] = mr[cell];
        gr_mi[g] = mi[cell];
        gr_d[g] = shapes[s];
      }
    }
    if ((rc = tmx_batch_upload(ctx, ng, gr_r.data(), gr_l.data(), gr_mr.data(),
                               gr_mi.data(), gr_d.data(), &S)) ||
        (rc = tmx_batch_compute(ctx))) {
      return rc;
    }
    if (grain_status) {
      for (int64_t g = 0; g < ng; ++g) {
        grain_status[c0 * nshape + g] = ctx->status_h[g];
      }
    }
    // ---- per-grain observable descriptors
    int nmax_chunk = 1;
    std::vector<TmxObsGrain> og(ng);
    int64_t t_total = 0;
    for (int64_t g = 0; g < ng; ++g) {
      const int64_t cell = c0 + g / nshape;
      const int64_t isz = (cell / nlambda) % nsizes;
      const int s = (int)(g % nshape);
      og[g].nmax = ctx->nmax_h[g];
      og[g].coef_set = orient_set[isz * nshape + s];
      og[g].t_off = ctx->t_off_h[g];
      og[g].k = 2. * M_PI / lambdas[cell % nlambda];
      og[g].r_ev = sizes[isz];
      nmax_chunk = std::max(nmax_chunk, og[g].nmax);
      if (og[g].nmax > 0) {
        t_total = std::max<int64_t>(t_total, og[g].t_off + tmx_tmatrix_size(og[g].nmax));
      }
      if (og[g].coef_set >= 0 && 2 * og[g].nmax + 1 > ncoef) {
        return fail(ctx, TMX_ERR_INVALID,
                    "tmx_get_table: orientation coefficients shorter than 2 nmax + 1");
      }
    }
    if ((rc = tmx_ensure_cg(ctx, nmax_chunk))) {
      return rc;
    }
    if ((rc = ensure(ctx, ctx->o_og, ng * sizeof(TmxObsGrain)))) {
      return rc;
    }
    ++ctx->plan_seq; // the observable buffers change below
    CK(cudaMemcpyAsync(ctx->o_og.p, og.data(), ng * sizeof(TmxObsGrain),
                       cudaMemcpyHostToDevice, st));
    // ---- amplitude jobs
    std::vector<TmxSJob> sj;
    std::vector<TmxQJob> qj;
    int64_t sidx = 0;
    const int64_t sca_base = ng * ntheta * (1 + (account ? (int64_t)ngauss * ngauss : 0));
    for (int64_t g = 0; g < ng; ++g) {
      if (og[g].nmax <= 0) {
        continue;
      }
      for (int t = 0; t < ntheta; ++t) {
        TmxQJob q;
        q.grain = (int32_t)g;
        q.pad = 0;
        q.out = g * ntheta + t;
        TmxSJob j;
        j.grain = (int32_t)g;
        j.angle_in = t;
        j.angle_out = t;
        j.nphi = 1;
        j.phi0 = 0;
        j.out = sidx;
        q.s_main = sidx;
        sidx += 1;
        sj.push_back(j);
        q.s_acc = sidx;
        if (account) {
          for (int ti = 0; ti < ngauss; ++ti) {
            TmxSJob a;
            a.grain = (int32_t)g;
            a.angle_in = acc_a0 + ti;
            a.angle_out = t;
            a.nphi = ngauss;
            a.phi0 = acc_p0;
            a.out = sidx;
            sidx += ngauss;
            sj.push_back(a);
          }
        }
        qj.push_back(q);
      }
    }
    int64_t nsca = 0;
    if (do_sca) {
      for (int64_t g = 0; g < ng; ++g) {
        for (int t = 0; t < ntheta; ++t) {
          if (og[g].nmax > 0) {
            TmxSJob j;
            j.grain = (int32_t)g;
            j.angle_in = sca_ain;
            j.angle_out = sca_a0 + t;
            j.nphi = nphi_sca;
            j.phi0 = sca_p0;
            j.out = sca_base + (g * ntheta + t) * nphi_sca;
            sj.push_back(j);
          }
        }
      }
      nsca = ng * ntheta * nphi_sca;
    }
    const int64_t s_total = sca_base + nsca;
    if ((rc = ensure(ctx, ctx->o_sj, std::max<size_t>(1, sj.size()) * sizeof(TmxSJob))) ||
        (rc = ensure(ctx, ctx->o_qj, std::max<size_t>(1, qj.size()) * sizeof(TmxQJob))) ||
        (rc = ensure(ctx, ctx->o_S, std::max<int64_t>(1, s_total) * 4 * sizeof(cplx))) ||
        (rc = ensure(ctx, ctx->o_gq, std::max<int64_t>(1, ng * ntheta * nq) * sizeof(double))) ||
        (rc = ensure(ctx, ctx->o_gz, std::max<int64_t>(1, do_sca ? nsca * 16 : 1) * sizeof(double))) ||
        (rc = ensure(ctx, ctx->o_cq, std::max<int64_t>(1, nc * ntheta * nq) * sizeof(double))) ||
        (rc = ensure(ctx, ctx->o_cz, std::max<int64_t>(1, do_sca ? nc * ntheta * nphi_sca * 16 : 1) * sizeof(double)))) {
      return rc;
    }
    if (!sj.empty()) {
      CK(cudaMemcpyAsync(ctx->o_sj.p, sj.data(), sj.size() * sizeof(TmxSJob),
                         cudaMemcpyHostToDevice, st));
    }
    if (!qj.empty()) {
      CK(cudaMemcpyAsync(ctx->o_qj.p, qj.data(), qj.size() * sizeof(TmxQJob),
                         cudaMemcpyHostToDevice, st));
    }
    if ((rc = upload_obs_plan(ctx, og, sj)) ||
        (ctx->obs_s_valid = false, false) ||
        (rc = run_amplitudes(ctx, (const cplx *)ctx->T.p, t_total, ncoef,
                             (cplx *)ctx->o_S.p, s_total))) {
      return rc;
    }
    if (nq > 0) {
      CK(cudaMemsetAsync(ctx->o_gq.p, 0, ng * ntheta * nq * sizeof(double), st));
      tmx_launch_q_epilogue((const TmxQJob *)ctx->o_qj.p, (int)qj.size(),
                            (const TmxObsGrain *)ctx->o_og.p, (const cplx *)ctx->o_S.p,
                            (const double *)ctx->o_wts.p, account ? ngauss : 0,
                            (double *)ctx->o_gq.p, nq, do_abs, do_ext, st);
      LAUNCHED();
      cudaEvent_t pe = nullptr;
      if ((rc = prof_begin(ctx, TMX_PROF_SHAPE_AVG, &pe))) {
        return rc;
      }
      tmx_launch_shape_avg((int)nc, nshape, ntheta * nq, (const double *)ctx->o_gq.p,
                           (const double *)ctx->o_shw.p, (double *)ctx->o_cq.p, st);
      LAUNCHED();
      // per cell: nshape inputs and one output per coefficient, the weights
      if ((rc = prof_end(ctx, TMX_PROF_SHAPE_AVG, pe, 0., st,
                         8. * (nc * (nshape + 1.) * ntheta * nq + nshape)))) {
        return rc;
      }
      CK(cudaMemcpyAsync(out_q + c0 * ntheta * nq, ctx->o_cq.p,
                         nc * ntheta * nq * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    if (do_sca) {
      tmx_launch_z_epilogue((int)nsca, (const cplx *)ctx->o_S.p + sca_base * 4,
                            (double *)ctx->o_gz.p, st);
      LAUNCHED();
      cudaEvent_t pz = nullptr;
      if ((rc = prof_begin(ctx, TMX_PROF_SHAPE_AVG, &pz))) {
        return rc;
      }
      tmx_launch_shape_avg((int)nc, nshape, ntheta * nphi_sca * 16,
                           (const double *)ctx->o_gz.p, (const double *)ctx->o_shw.p,
                           (double *)ctx->o_cz.p, st);
      LAUNCHED();
      if ((rc = prof_end(ctx, TMX_PROF_SHAPE_AVG, pz, 0., st,
                         8. * (nc * (nshape + 1.) * ntheta * nphi_sca * 16 + nshape)))) {
        return rc;
      }
      CK(cudaMemcpyAsync(out_z + c0 * ntheta * nphi_sca * 16, ctx->o_cz.p,
                         nc * ntheta * nphi_sca * 16 * sizeof(double),
                         cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    c0 = c1;
  }
  return TMX_OK;
}

// Clebsch-Gordan table for every (n1, n2) up to nmax (cached; rebuilt when a
// larger nmax is needed)
int tmx_ensure_cg(tmx_ctx *ctx, int nmax) {
  if (ctx->cg_nmax >= nmax && ctx->cg_nmax > 0) {
    return TMX_OK;
  }
  nmax = std::max(nmax, ctx->cg_nmax);
  cudaStream_t st = ctx->stream;
  std::vector<int64_t> off((size_t)nmax * nmax);
  int64_t tot = 0;
  for (int n1 = 1; n1 <= nmax; ++n1) {
    for (int n2 = 1; n2 <= nmax; ++n2) {
      const int M = std::min(n1, n2);
      off[(size_t)(n1 - 1) * nmax + (n2 - 1)] = tot;
      tot += (int64_t)(2 * M + 1) * (M + 1);
    }
  }
  const int blocks = 4 * 148;
  int rc;
  if ((rc = ensure(ctx, ctx->cg, tot * sizeof(double))) ||
      (rc = ensure(ctx, ctx->cg_off, off.size() * sizeof(int64_t))) ||
      (rc = ensure(ctx, ctx->o_work,
                   (size_t)blocks * 128 * 2 * (2 * nmax + 1) * sizeof(double)))) {
    return rc;
  }
  CK(cudaMemcpyAsync(ctx->cg_off.p, off.data(), off.size() * sizeof(int64_t),
                     cudaMemcpyHostToDevice, st));
  tmx_launch_cg(nmax, (const int64_t *)ctx->cg_off.p, (double *)ctx->cg.p,
                (double *)ctx->o_work.p, blocks, st);
  LAUNCHED();
  CK(cudaStreamSynchronize(st));
  ctx->cg_nmax = nmax;
  return TMX_OK;
}

// ------------------------------------------- per-grain observables / grads --

namespace {

// orientation-averaged theta -> theta amplitudes of every grain of the last
// batch for the T-matrices at `Tsrc`; S[(grain * ntheta + t) * 4]
int batch_amplitudes(tmx_ctx *ctx, const cplx *Tsrc, int ntheta, int ncoef,
                     cplx *S_out) {
  return run_amplitudes(ctx, Tsrc, ctx->p2_t_total, ncoef, S_out,
                        ctx->n * ntheta);
}

// descriptors shared by the per-grain observable and gradient passes
int batch_observable_setup(tmx_ctx *ctx, int ntheta, const double *thetas,
                           const double *coeffs, int ncoef) {
  cudaStream_t st = ctx->stream;
  const int64_t n = ctx->n;
  int rc;
  // the plan of the previous call, if nothing it depends on has changed
  // since (the observables of a batch followed by its gradients)
  tmx_ctx::ObsKey &key = ctx->obs_key;
  if (key.valid && key.batch_seq == ctx->batch_seq && key.plan_seq == ctx->plan_seq &&
      key.has_coeffs == (coeffs != nullptr) && (int)key.thetas.size() == ntheta &&
      std::equal(key.thetas.begin(), key.thetas.end(), thetas) &&
      (!coeffs || ((int)key.coeffs.size() == ncoef &&
                   std::equal(key.coeffs.begin(), key.coeffs.end(), coeffs)))) {
    return TMX_OK;
  }
  key.valid = false;
  ctx->obs_s_valid = false;
  std::vector<TmxAngle> ang(ntheta);
  for (int i = 0; i < ntheta; ++i) {
    ang[i] = make_angle(cos(thetas[i]));
  }
  std::vector<cplx> phis(1, mkc(1., 0.));
  std::vector<TmxObsGrain> og(n);
  std::vector<TmxSJob> sj;
  std::vector<TmxQJob> qj;
  sj.reserve((size_t)n * ntheta);
  qj.reserve((size_t)n * ntheta);
  for (int64_t g = 0; g < n; ++g) {
    og[g].nmax = ctx->nmax_h[g];
    og[g].coef_set = coeffs ? 0 : -1;
    og[g].t_off = ctx->t_off_h[g];
    og[g].k = ctx->up_grains[g].k;
    og[g].r_ev = ctx->up_grains[g].r_ev;
    if (coeffs && 2 * og[g].nmax + 1 > ncoef) {
      return fail(ctx, TMX_ERR_INVALID,
                  "orientation coefficients shorter than 2 nmax + 1");
    }
    if (og[g].nmax <= 0) {
      continue;
    }
    for (int t = 0; t < ntheta; ++t) {
      TmxSJob j;
      j.grain = (int32_t)g;
      j.angle_in = t;
      j.angle_out = t;
      j.nphi = 1;
      j.phi0 = 0;
      j.out = g * ntheta + t;
      sj.push_back(j);
      TmxQJob q;
      q.grain = (int32_t)g;
      q.pad = 0;
      q.out = g * ntheta + t;
      q.s_main = g * ntheta + t;
      q.s_acc = 0;
      qj.push_back(q);
    }
  }
  if ((rc = ensure(ctx, ctx->o_angles, std::max(1, ntheta) * sizeof(TmxAngle))) ||
      (rc = ensure(ctx, ctx->o_phis, sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->o_og, std::max<int64_t>(1, n) * sizeof(TmxObsGrain))) ||
      (rc = ensure(ctx, ctx->o_sj, std::max<size_t>(1, sj.size()) * sizeof(TmxSJob))) ||
      (rc = ensure(ctx, ctx->o_qj, std::max<size_t>(1, qj.size()) * sizeof(TmxQJob))) ||
      (rc = ensure(ctx, ctx->o_coef, std::max(1, ncoef) * sizeof(double)))) {
    return rc;
  }
  CK(cudaMemcpyAsync(ctx->o_angles.p, ang.data(), ntheta * sizeof(TmxAngle),
                     cudaMemcpyHostToDevice, st));
  ctx->o_nangles = ntheta;
  CK(cudaMemcpyAsync(ctx->o_phis.p, phis.data(), sizeof(cplx),
                     cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->o_og.p, og.data(), n * sizeof(TmxObsGrain),
                     cudaMemcpyHostToDevice, st));
  if (!sj.empty()) {
    CK(cudaMemcpyAsync(ctx->o_sj.p, sj.data(), sj.size() * sizeof(TmxSJob),
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->o_qj.p, qj.data(), qj.size() * sizeof(TmxQJob),
                       cudaMemcpyHostToDevice, st));
  }
  if (coeffs) {
    CK(cudaMemcpyAsync(ctx->o_coef.p, coeffs, ncoef * sizeof(double),
                       cudaMemcpyHostToDevice, st));
  }
  ctx->o_nsj = (int)sj.size();
  ctx->o_nqj = (int)qj.size();
  if (coeffs) {
    int nmax_b = 1;
    for (int64_t g = 0; g < n; ++g) {
      nmax_b = std::max(nmax_b, og[g].nmax);
    }
    if ((rc = tmx_ensure_cg(ctx, nmax_b))) {
      return rc;
    }
  }
  if ((rc = upload_obs_plan(ctx, og, sj))) {
    return rc;
  }
  key.valid = true;
  key.batch_seq = ctx->batch_seq;
  key.plan_seq = ctx->plan_seq;
  key.thetas.assign(thetas, thetas + ntheta);
  key.has_coeffs = coeffs != nullptr;
  if (coeffs) {
    key.coeffs.assign(coeffs, coeffs + ncoef);
  } else {
    key.coeffs.clear();
  }
  return TMX_OK;
}

} // namespace

extern "C" int tmx_batch_observables(tmx_ctx *ctx, int32_t ntheta,
                                     const double *thetas, const double *coeffs,
                                     int32_t ncoef, double *q) {
  if (!ctx || ntheta < 1 || !thetas || !q) {
    return TMX_ERR_INVALID;
  }
  if (!ctx->have_batch) {
    return fail(ctx, TMX_ERR_STATE, "no batch has been computed");
  }
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int64_t n = ctx->n;
  int rc;
  if ((rc = batch_observable_setup(ctx, ntheta, thetas, coeffs, ncoef)) ||
      (rc = ensure(ctx, ctx->o_S, std::max<int64_t>(1, n * ntheta) * 4 * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->o_gq, std::max<int64_t>(1, n * ntheta * 3) * sizeof(double)))) {
    return rc;
  }
  ctx->obs_s_valid = false;
  if ((rc = batch_amplitudes(ctx, (const cplx *)ctx->T.p, ntheta, ncoef,
                             (cplx *)ctx->o_S.p))) {
    return rc;
  }
  ctx->obs_s_valid = true;
  CK(cudaMemsetAsync(ctx->o_gq.p, 0, n * ntheta * 3 * sizeof(double), st));
  tmx_launch_q_epilogue((const TmxQJob *)ctx->o_qj.p, ctx->o_nqj,
                        (const TmxObsGrain *)ctx->o_og.p, (const cplx *)ctx->o_S.p,
                        nullptr, 0, (double *)ctx->o_gq.p, 3, 0, 1, st);
  LAUNCHED();
  CK(cudaMemcpyAsync(q, ctx->o_gq.p, n * ntheta * 3 * sizeof(double),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return TMX_OK;
}

extern "C" int tmx_batch_gradients(tmx_ctx *ctx, int32_t ntheta,
                                   const double *thetas, const double *coeffs,
                                   int32_t ncoef, double *q, double *dq) {
  if (!ctx || ntheta < 1 || !thetas || !dq) {
    return TMX_ERR_INVALID;
  }
  if (!ctx->have_batch) {
    return fail(ctx, TMX_ERR_STATE, "no batch has been computed");
  }
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int64_t n = ctx->n;
  int rc;
  if (ctx->t_averaged) {
    return fail(ctx, TMX_ERR_STATE,
                "gradients need the batch's own T-matrices, not orientation averages");
  }
  // LU factors of every item: kept by the batch's block rounds, or by a
  // single-round batch in the p2 set; otherwise the forward blocks run again
  // in one round that keeps them
  if (!ctx->rounds_lu && ctx->p2_rounds > 1 && (rc = tmx_rerun_blocks(ctx))) {
    return rc;
  }
  struct RoundView {
    const TmxItem *items;
    const TmxSlot *slots;
    const double *tab, *nsc;
    cplx *lu;
    std::vector<std::array<int64_t, 3>> seg; // size buckets: [i0, i1), max class size
    int64_t scr;
  };
  // the class-size buckets of a round whose items are sorted by size,
  // largest first
  auto segments = [](const std::vector<int> &nb) {
    std::vector<std::array<int64_t, 3>> seg;
    const int edges[] = {1 << 30, 64, 32, 16, 8, 0};
    const int64_t nitems = (int64_t)nb.size();
    int64_t i0 = 0;
    for (int b = 0; b < 5; ++b) {
      int64_t i1 = i0;
      int mx = 0;
      while (i1 < nitems && nb[i1] > edges[b + 1]) {
        mx = std::max(mx, nb[i1]);
        ++i1;
      }
      if (i1 > i0) {
        seg.push_back({i0, i1, (int64_t)mx});
      }
      i0 = i1;
    }
    return seg;
  };
  std::vector<RoundView> views;
  if (ctx->rounds_lu) {
    for (const auto &r : ctx->rounds_kept) {
      views.push_back({r.items, r.slots, r.tab, r.nsc, r.lu,
                       r.seg.empty() ? segments(r.nb) : r.seg, r.scr_total});
    }
  } else {
    if ((rc = ensure(ctx, ctx->lu, std::max<int64_t>(1, ctx->p2_scr_total) * sizeof(cplx)))) {
      return rc;
    }
    views.push_back({(const TmxItem *)ctx->p2items.p, (const TmxSlot *)ctx->p2slots.p,
                     (const double *)ctx->p2tab.p, (const double *)ctx->p2nsc.p,
                     (cplx *)ctx->lu.p, segments(ctx->p2_nb), ctx->p2_scr_total});
  }
  // each round's tangent scratch in its own region: the rounds' size
  // buckets run concurrently
  int64_t scr_sum = 1;
  for (const RoundView &v : views) {
    scr_sum += v.scr;
  }
  const int64_t tt = ctx->p2_t_total;
  NvtxRange range("tmx_gradients");
  if ((rc = ensure(ctx, ctx->tscr, 3 * scr_sum * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->dT, std::max<int64_t>(1, 3 * tt) * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->dS, std::max<int64_t>(1, 4 * n * ntheta) * 4 * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->o_gq, std::max<int64_t>(1, n * ntheta * 3) * sizeof(double))) ||
      (rc = ensure(ctx, ctx->o_gz, std::max<int64_t>(1, n * ntheta * 12) * sizeof(double)))) {
    return rc;
  }
  CK(cudaMemsetAsync(ctx->dT.p, 0, std::max<int64_t>(1, 3 * tt) * sizeof(cplx), st));
  // every (round, size bucket) launch may start once dT is cleared: they
  // write disjoint blocks of dT and disjoint scratch, so they run on the
  // library stream and the eight others side by side and join before the
  // observables
  cudaStream_t gstreams[9] = {st,          ctx->aux[0], ctx->aux[1],
                              ctx->aux[2], ctx->aux[3], ctx->aux[4],
                              ctx->aux[5], ctx->stream2, ctx->stream3};
  cudaEvent_t gfork;
  CK(cudaEventCreateWithFlags(&gfork, cudaEventDisableTiming));
  CK(cudaEventRecord(gfork, st));
  bool gused[9] = {true, false, false, false, false, false, false, false, false};
  int glaunch = 0;
  int64_t scr_off = 0;
  for (const RoundView &v : views) {
    for (const auto &sg : v.seg) {
      const int64_t i0 = sg[0], i1 = sg[1];
      const int max_nb = (int)sg[2];
      {
        const int gi = glaunch++ % 9;
        cudaStream_t gs = gstreams[gi];
        if (!gused[gi]) {
          CK(cudaStreamWaitEvent(gs, gfork, 0));
          gused[gi] = true;
        }
        if (!ctx->rounds_lu && !ctx->lu_ready) {
          TmxBlockArgs B;
          B.items = v.items + i0;
          B.nitems = (int)(i1 - i0);
          B.slots = v.slots;
          B.grains = (const TmxGrain *)ctx->grains.p;
          B.tab = v.tab;
          B.nsc = v.nsc;
          B.wig = (const double *)ctx->wig.p;
          B.wig_off = (const int64_t *)ctx->wig_off.p;
          B.scratch = (cplx *)ctx->p2scratch.p;
          B.tout = (cplx *)ctx->T.p;
          B.diag = nullptr;
          B.status = (int32_t *)ctx->status.p;
          B.max_nb = max_nb;
          B.chunk_nodes = tmx_host_chunk_nodes(max_nb);
          B.family = dispatch_family(ctx, max_nb);
          B.lu = v.lu;
          tmx_launch_blocks(B, gs);
          LAUNCHED();
        }
        TmxTangentArgs A;
        A.items = v.items + i0;
        A.nitems = (int)(i1 - i0);
        A.nparams = 3;
        A.slots = v.slots;
        A.grains = (const TmxGrain *)ctx->grains.p;
        A.tab = v.tab;
        A.nsc = v.nsc;
        A.wig = (const double *)ctx->wig.p;
        A.wig_off = (const int64_t *)ctx->wig_off.p;
        A.lu = v.lu;
        A.T = (const cplx *)ctx->T.p;
        A.scratch = (cplx *)ctx->tscr.p + 3 * scr_off;
        A.scratch_stride = v.scr;
        A.dT = (cplx *)ctx->dT.p;
        A.dT_stride = tt;
        A.chunk_nodes = std::max(1, tmx_host_chunk_nodes(max_nb) / 2);
        A.max_nb = max_nb;
        cudaEvent_t pe = nullptr;
        if ((rc = prof_begin(ctx, TMX_PROF_TANGENTS, &pe, gs))) {
          return rc;
        }
        tmx_launch_tangents(A, gs);
        LAUNCHED();
        if ((rc = prof_end(ctx, TMX_PROF_TANGENTS, pe, 0., gs, 0., A.nitems))) {
          return rc;
        }
      }
    }
    scr_off += v.scr;
  }
  for (int gi = 1; gi < 9; ++gi) {
    if (gused[gi]) {
      CK(cudaEventRecord(gfork, gstreams[gi]));
      CK(cudaStreamWaitEvent(st, gfork, 0));
    }
  }
  CK(cudaEventDestroy(gfork));
  if ((rc = batch_observable_setup(ctx, ntheta, thetas, coeffs, ncoef))) {
    return rc;
  }
  cplx *S = (cplx *)ctx->dS.p;
  const int64_t sz = n * ntheta * 4;
  // the T-matrices' own amplitudes: those of tmx_batch_observables when it
  // ran on this batch with the same plan (still in o_S), else computed here
  const bool have_s = ctx->obs_s_valid;
  const cplx *S0 = have_s ? (const cplx *)ctx->o_S.p : S;
  {
    // the three tangents (and T) in one pass (shared angle and coupling work)
    const cplx *src[4] = {(const cplx *)ctx->T.p, (const cplx *)ctx->dT.p,
                          (const cplx *)ctx->dT.p + tt, (const cplx *)ctx->dT.p + 2 * tt};
    cplx *dst[4] = {S, S + sz, S + 2 * sz, S + 3 * sz};
    const int k0 = have_s ? 1 : 0;
    if ((rc = run_amplitudes(ctx, src + k0, 4 - k0, ctx->p2_t_total, ncoef, dst + k0,
                             n * ntheta))) {
      return rc;
    }
  }
  CK(cudaMemsetAsync(ctx->o_gq.p, 0, n * ntheta * 3 * sizeof(double), st));
  CK(cudaMemsetAsync(ctx->o_gz.p, 0, n * ntheta * 12 * sizeof(double), st));
  tmx_launch_q_epilogue((const TmxQJob *)ctx->o_qj.p, ctx->o_nqj,
                        (const TmxObsGrain *)ctx->o_og.p, S0, nullptr, 0,
                        (double *)ctx->o_gq.p, 3, 0, 1, st);
  LAUNCHED();
  tmx_launch_dq_epilogue((const TmxQJob *)ctx->o_qj.p, ctx->o_nqj,
                         (const TmxObsGrain *)ctx->o_og.p, S0, S + sz, S + 2 * sz,
                         S + 3 * sz, (double *)ctx->o_gz.p, st);
  LAUNCHED();
  if (q) {
    CK(cudaMemcpyAsync(q, ctx->o_gq.p, n * ntheta * 3 * sizeof(double),
                       cudaMemcpyDeviceToHost, st));
  }
  CK(cudaMemcpyAsync(dq, ctx->o_gz.p, n * ntheta * 12 * sizeof(double),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return TMX_OK;
}

// ------------------------------------------ plain-path observables (A25) --

namespace {

// Lab-frame direction (theta, phi) in the frame of a particle whose symmetry
// axis points at (beta, alpha), and the 2 x 2 amplitude rotation between the
// frames (TMatrix::get_forward_scattering_matrix, TMatrix.hpp:1306-1420).
struct PDir {
  TmxAngle a;        // cos, sin, 1/sin (or 9000) of the particle zenith
  double cphi, sphi; // particle azimuth
  double R[2][2];    // AP B AL
};

PDir particle_dir(double cosalpha, double sinalpha, double cosbeta,
                  double sinbeta, double theta, double phi) {
  PDir d;
  const double ct = cos(theta), st = sin(theta);
  const double cp = cos(phi), sp = sin(phi);
  const double cosphirel = cp * cosalpha + sp * sinalpha;
  const double sinphirel = sp * cosalpha - cp * sinalpha;
  const double ctp = ct * cosbeta + st * sinbeta * cosphirel;
  const double stp = sin(acos(ctp));
  double cphi, sphi, sinv;
  if (stp != 0.) {
    sinv = 1. / stp;
    cphi = (cosbeta * st * cosphirel - sinbeta * ct) * sinv;
    sphi = st * sinphirel * sinv;
  } else {
    cphi = 1.;
    sphi = 0.;
    sinv = 9000.;
  }
  d.a.c = ctp;
  d.a.s = stp;
  d.a.si = sinv;
  d.cphi = cphi;
  d.sphi = sphi;
  const double B[3][3] = {{cosalpha * cosbeta, sinalpha * cosbeta, -sinbeta},
                          {-sinalpha, cosalpha, 0.},
                          {cosalpha * sinbeta, sinalpha * sinbeta, cosbeta}};
  const double AL[3][2] = {{ct * cp, -sp}, {ct * sp, cp}, {-st, 0.}};
  const double AP[2][3] = {{ctp * cphi, ctp * sphi, -stp}, {-sphi, cphi, 0.}};
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
      d.R[i][j] = 0.;
      for (int k = 0; k < 3; ++k) {
        d.R[i][j] += AP[i][k] * C[k][j];
      }
    }
  }
  return d;
}

// direction of a particle-frame zenith angle without rotation (the
// four-angle form of get_forward_scattering_matrix, TMatrix.hpp:1245-1290)
TmxAngle plain_angle(double theta) {
  TmxAngle a;
  a.c = cos(theta);
  a.s = sin(theta);
  a.si = (a.s != 0.) ? 1. / a.s : 9000.;
  return a;
}

typedef std::complex<double> zc;

// Z from the 2 x 2 amplitude matrix S (TMatrix.hpp:1896-1948), row major
void z_from_s(const zc S[2][2], double *Z) {
  const zc ic(0., 1.);
  const double half(0.5);
  Z[0] = (half * (S[0][0] * conj(S[0][0]) + S[0][1] * conj(S[0][1]) +
                  S[1][0] * conj(S[1][0]) + S[1][1] * conj(S[1][1])))
             .real();
  Z[1] = (half * (S[0][0] * conj(S[0][0]) - S[0][1] * conj(S[0][1]) +
                  S[1][0] * conj(S[1][0]) - S[1][1] * conj(S[1][1])))
             .real();
  Z[2] = (-S[0][0] * conj(S[0][1]) - S[1][1] * conj(S[1][0])).real();
  Z[3] = (ic * (S[0][0] * conj(S[0][1]) - S[1][1] * conj(S[1][0]))).real();
  Z[4] = (half * (S[0][0] * conj(S[0][0]) + S[0][1] * conj(S[0][1]) -
                  S[1][0] * conj(S[1][0]) - S[1][1] * conj(S[1][1])))
             .real();
  Z[5] = (half * (S[0][0] * conj(S[0][0]) - S[0][1] * conj(S[0][1]) -
                  S[1][0] * conj(S[1][0]) + S[1][1] * conj(S[1][1])))
             .real();
  Z[6] = (-S[0][0] * conj(S[0][1]) + S[1][1] * conj(S[1][0])).real();
  Z[7] = (ic * (S[0][0] * conj(S[0][1]) + S[1][1] * conj(S[1][0]))).real();
  Z[8] = (-S[0][0] * conj(S[1][0]) - S[1][1] * conj(S[0][1])).real();
  Z[9] = (-S[0][0] * conj(S[1][0]) + S[1][1] * conj(S[0][1])).real();
  Z[10] = (S[0][0] * conj(S[1][1]) + S[0][1] * conj(S[1][0])).real();
  Z[11] = (-ic * (S[0][0] * conj(S[1][1]) + S[1][0] * conj(S[0][1]))).real();
  Z[12] = (ic * (S[1][0] * conj(S[0][0]) + S[1][1] * conj(S[0][1]))).real();
  Z[13] = (ic * (S[1][0] * conj(S[0][0]) - S[1][1] * conj(S[0][1]))).real();
  Z[14] = (-ic * (S[1][1] * conj(S[0][0]) - S[0][1] * conj(S[1][0]))).real();
  Z[15] = (S[1][1] * conj(S[0][0]) - S[0][1] * conj(S[1][0])).real();
}

// K from the forward amplitude matrix (TMatrix.hpp:1972-2010), row major
void k_from_s(double k, const zc S[2][2], double *K) {
  const double pf = 2. * M_PI / k;
  for (int i = 0; i < 16; ++i) {
    K[i] = 0.;
  }
  K[0] = pf * (S[0][0] + S[1][1]).imag();
  K[5] = K[0];
  K[10] = K[0];
  K[15] = K[0];
  K[1] = pf * (S[0][0] - S[1][1]).imag();
  K[4] = K[1];
  K[2] = -pf * (S[0][1] + S[1][0]).imag();
  K[8] = K[2];
  K[3] = pf * (S[1][0] - S[0][1]).real();
  K[12] = K[3];
  K[6] = pf * (S[1][0] - S[0][1]).imag();
  K[9] = -K[6];
  K[7] = -pf * (S[0][1] + S[1][0]).real();
  K[13] = -K[7];
  K[11] = pf * (S[1][1] - S[0][0]).real();
  K[14] = -K[11];
}

// Amplitude matrices S^P of jobs (grain, incoming angle index, outgoing
// angle index, e^{i(phi_out - phi_in)}) for the T-matrices of the last batch
// (plain or averaged): sorted by grain for the amplitude kernel's groups,
// results in job order.
int plain_amplitudes(tmx_ctx *ctx, const std::vector<int32_t> &grain,
                     const std::vector<TmxAngle> &ang,
                     const std::vector<int32_t> &ain,
                     const std::vector<int32_t> &aout,
                     const std::vector<cplx> &e1, std::vector<zc> &S) {
  cudaStream_t st = ctx->stream;
  const int64_t n = ctx->n;
  const int64_t nj = (int64_t)grain.size();
  int rc;
  std::vector<TmxObsGrain> og(n);
  for (int64_t g = 0; g < n; ++g) {
    og[g].nmax = ctx->nmax_h[g];
    og[g].coef_set = -1;
    og[g].t_off = ctx->t_off_h[g];
    og[g].k = ctx->up_grains[g].k;
    og[g].r_ev = ctx->up_grains[g].r_ev;
  }
  std::vector<int64_t> order(nj);
  for (int64_t j = 0; j < nj; ++j) {
    order[j] = j;
  }
  std::stable_sort(order.begin(), order.end(),
                   [&](int64_t a, int64_t b) { return grain[a] < grain[b]; });
  std::vector<TmxSJob> sj;
  sj.reserve(nj);
  for (int64_t q = 0; q < nj; ++q) {
    const int64_t j = order[q];
    if (og[grain[j]].nmax <= 0) {
      continue;
    }
    TmxSJob J;
    J.grain = grain[j];
    J.angle_in = ain[j];
    J.angle_out = aout[j];
    J.nphi = 1;
    J.phi0 = j;
    J.out = j;
    sj.push_back(J);
  }
  if ((rc = ensure(ctx, ctx->o_og, std::max<int64_t>(1, n) * sizeof(TmxObsGrain))) ||
      (rc = ensure(ctx, ctx->o_angles, std::max<size_t>(1, ang.size()) * sizeof(TmxAngle))) ||
      (rc = ensure(ctx, ctx->o_phis, std::max<size_t>(1, e1.size()) * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->o_sj, std::max<size_t>(1, sj.size()) * sizeof(TmxSJob))) ||
      (rc = ensure(ctx, ctx->o_S, std::max<int64_t>(1, nj) * 4 * sizeof(cplx)))) {
    return rc;
  }
  ++ctx->plan_seq; // the observable buffers change below
  CK(cudaMemcpyAsync(ctx->o_og.p, og.data(), n * sizeof(TmxObsGrain),
                     cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->o_angles.p, ang.data(), ang.size() * sizeof(TmxAngle),
                     cudaMemcpyHostToDevice, st));
  ctx->o_nangles = (int)ang.size();
  CK(cudaMemcpyAsync(ctx->o_phis.p, e1.data(), e1.size() * sizeof(cplx),
                     cudaMemcpyHostToDevice, st));
  if (!sj.empty()) {
    CK(cudaMemcpyAsync(ctx->o_sj.p, sj.data(), sj.size() * sizeof(TmxSJob),
                       cudaMemcpyHostToDevice, st));
  }
  if ((rc = upload_obs_plan(ctx, og, sj)) ||
      (ctx->obs_s_valid = false, false) ||
      (rc = run_amplitudes(ctx, (const cplx *)ctx->T.p, ctx->p2_t_total, 1,
                           (cplx *)ctx->o_S.p, nj))) {
    return rc;
  }
  std::vector<cplx> Sh(4 * nj);
  CK(cudaMemcpyAsync(Sh.data(), ctx->o_S.p, 4 * nj * sizeof(cplx),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  S.resize(4 * nj);
  for (int64_t i = 0; i < 4 * nj; ++i) {
    S[i] = zc(Sh[i].x, Sh[i].y);
  }
  return TMX_OK;
}

int check_jobs(tmx_ctx *ctx, int64_t njobs, const int64_t *grain) {
  if (!ctx->have_batch) {
    return fail(ctx, TMX_ERR_STATE, "no batch has been computed");
  }
  for (int64_t j = 0; j < njobs; ++j) {
    if (grain[j] < 0 || grain[j] >= ctx->n) {
      return fail(ctx, TMX_ERR_INVALID, "grain index out of range");
    }
  }
  return TMX_OK;
}

// lab-frame S for jobs at particle orientations: S^L = R_out^-1 S^P R_in
// (TMatrix.hpp:1420-1460)
int lab_amplitudes(tmx_ctx *ctx, int64_t njobs, const int64_t *grain,
                   const double *alpha, const double *beta,
                   const double *theta_in, const double *phi_in,
                   const double *theta_out, const double *phi_out,
                   std::vector<zc> &SL) {
  std::vector<int32_t> g(njobs), ain(njobs), aout(njobs);
  std::vector<TmxAngle> ang(2 * njobs);
  std::vector<cplx> e1(njobs);
  std::vector<PDir> din(njobs), dout(njobs);
  for (int64_t j = 0; j < njobs; ++j) {
    const double ca = cos(alpha[j]), sa = sin(alpha[j]);
    const double cb = cos(beta[j]), sb = sin(beta[j]);
    din[j] = particle_dir(ca, sa, cb, sb, theta_in[j], phi_in[j]);
    dout[j] = particle_dir(ca, sa, cb, sb, theta_out[j], phi_out[j]);
    g[j] = (int32_t)grain[j];
    ang[2 * j] = din[j].a;
    ang[2 * j + 1] = dout[j].a;
    ain[j] = (int32_t)(2 * j);
    aout[j] = (int32_t)(2 * j + 1);
    e1[j] = mkc(dout[j].cphi * din[j].cphi + dout[j].sphi * din[j].sphi,
                dout[j].sphi * din[j].cphi - dout[j].cphi * din[j].sphi);
  }
  std::vector<zc> SP;
  int rc = plain_amplitudes(ctx, g, ang, ain, aout, e1, SP);
  if (rc) {
    return rc;
  }
  SL.resize(4 * njobs);
  for (int64_t j = 0; j < njobs; ++j) {
    const zc *S = SP.data() + 4 * j;
    const double(&Ri)[2][2] = din[j].R;
    double Ro[2][2];
    const double det = 1. / (dout[j].R[0][0] * dout[j].R[1][1] -
                             dout[j].R[0][1] * dout[j].R[1][0]);
    Ro[0][0] = dout[j].R[1][1] * det;
    Ro[0][1] = -dout[j].R[0][1] * det;
    Ro[1][0] = -dout[j].R[1][0] * det;
    Ro[1][1] = dout[j].R[0][0] * det;
    const zc cS11 = S[0] * Ri[0][0] + S[1] * Ri[1][0];
    const zc cS12 = S[0] * Ri[0][1] + S[1] * Ri[1][1];
    const zc cS21 = S[2] * Ri[0][0] + S[3] * Ri[1][0];
    const zc cS22 = S[2] * Ri[0][1] + S[3] * Ri[1][1];
    SL[4 * j + 0] = Ro[0][0] * cS11 + Ro[0][1] * cS21;
    SL[4 * j + 1] = Ro[0][0] * cS12 + Ro[0][1] * cS22;
    SL[4 * j + 2] = Ro[1][0] * cS11 + Ro[1][1] * cS21;
    SL[4 * j + 3] = Ro[1][0] * cS12 + Ro[1][1] * cS22;
  }
  return TMX_OK;
}

// absorption cross sections (Cabs, Cabspol) of one grain at zenith angles
// th: per angle the forward amplitude and ngauss^2 incoming directions
// (TMatrix.hpp:2133-2200)
int absorption(tmx_ctx *ctx, int32_t grain, int32_t ntheta, const double *th,
               int32_t ngauss, double *out) {
  std::vector<double> ct(ngauss), wt(ngauss), ph(ngauss), wp(ngauss), tg(ngauss);
  tmx_host_gauss_legendre(ngauss, ct.data(), wt.data());
  gl_ab(ngauss, 0., 2. * M_PI, ph.data(), wp.data());
  for (int i = 0; i < ngauss; ++i) {
    tg[i] = acos(ct[i]);
  }
  std::vector<TmxAngle> ang;
  for (int i = 0; i < ngauss; ++i) {
    ang.push_back(plain_angle(tg[i]));
  }
  const int a0 = (int)ang.size();
  for (int t = 0; t < ntheta; ++t) {
    ang.push_back(plain_angle(th[t]));
  }
  std::vector<int32_t> g, ain, aout;
  std::vector<cplx> e1;
  for (int t = 0; t < ntheta; ++t) {
    g.push_back(grain);
    ain.push_back(a0 + t);
    aout.push_back(a0 + t);
    e1.push_back(mkc(1., 0.));
    for (int it = 0; it < ngauss; ++it) {
      for (int ip = 0; ip < ngauss; ++ip) {
        // e^{i(0 - phi_in)} as the reference forms it
        const double cp = cos(ph[ip]), sp = sin(ph[ip]);
        g.push_back(grain);
        ain.push_back(it);
        aout.push_back(a0 + t);
        e1.push_back(mkc(1. * cp + 0. * sp, 0. * cp - 1. * sp));
      }
    }
  }
  std::vector<zc> S;
  int rc = plain_amplitudes(ctx, g, ang, ain, aout, e1, S);
  if (rc) {
    return rc;
  }
  const double pf = 2. * M_PI / ctx->up_grains[grain].k;
  const double half(0.5);
  int64_t j = 0;
  for (int t = 0; t < ntheta; ++t) {
    const zc *s = S.data() + 4 * j++;
    double c0 = pf * (s[0] + s[3]).imag();
    double c1 = pf * (s[0] - s[3]).imag();
    for (int it = 0; it < ngauss; ++it) {
      for (int ip = 0; ip < ngauss; ++ip) {
        const zc *q = S.data() + 4 * j++;
        const double w = wt[it] * wp[ip];
        const double z00 = (half * (q[0] * conj(q[0]) + q[1] * conj(q[1]) +
                                    q[2] * conj(q[2]) + q[3] * conj(q[3])))
                               .real();
        const double z10 = (half * (q[0] * conj(q[0]) + q[1] * conj(q[1]) -
                                    q[2] * conj(q[2]) - q[3] * conj(q[3])))
                               .real();
        c0 -= z00 * w;
        c1 -= z10 * w;
      }
    }
    out[2 * t] = c0;
    out[2 * t + 1] = c1;
  }
  return TMX_OK;
}

} // namespace

extern "C" int tmx_batch_orientation_average(tmx_ctx *ctx, const double *coeffs,
                                             int32_t nsets, int32_t ncoef,
                                             const int32_t *coef_set) {
  if (!ctx || nsets < 0 || (nsets > 0 && (!coeffs || ncoef < 1))) {
    return TMX_ERR_INVALID;
  }
  if (!ctx->have_batch) {
    return fail(ctx, TMX_ERR_STATE, "no batch has been computed");
  }
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int64_t n = ctx->n;
  int rc;
  std::vector<TmxObsGrain> og(n);
  int nmax_b = 1;
  for (int64_t g = 0; g < n; ++g) {
    og[g].nmax = ctx->nmax_h[g];
    og[g].coef_set = coef_set ? coef_set[g] : -1;
    og[g].t_off = ctx->t_off_h[g];
    og[g].k = ctx->up_grains[g].k;
    og[g].r_ev = ctx->up_grains[g].r_ev;
    if (og[g].coef_set >= nsets) {
      return fail(ctx, TMX_ERR_INVALID, "orientation set index");
    }
    if (og[g].coef_set >= 0 && og[g].nmax > 0 && 2 * og[g].nmax + 1 > ncoef) {
      return fail(ctx, TMX_ERR_INVALID,
                  "orientation coefficients shorter than 2 nmax + 1");
    }
    nmax_b = std::max(nmax_b, og[g].nmax);
  }
  const int64_t t_total = ctx->p2_t_total;
  if ((rc = ensure(ctx, ctx->o_og, std::max<int64_t>(1, n) * sizeof(TmxObsGrain))) ||
      (rc = ensure(ctx, ctx->o_coef, std::max<int64_t>(1, (int64_t)nsets * ncoef) * sizeof(double))) ||
      (rc = ensure(ctx, ctx->Ta, std::max<int64_t>(1, t_total) * sizeof(cplx))) ||
      (rc = tmx_ensure_cg(ctx, nmax_b))) {
    return rc;
  }
  ++ctx->plan_seq; // the observable buffers change below
  CK(cudaMemcpyAsync(ctx->o_og.p, og.data(), n * sizeof(TmxObsGrain),
                     cudaMemcpyHostToDevice, st));
  if (nsets > 0) {
    CK(cudaMemcpyAsync(ctx->o_coef.p, coeffs, (int64_t)nsets * ncoef * sizeof(double),
                       cudaMemcpyHostToDevice, st));
  }
  if ((rc = upload_obs_plan(ctx, og, std::vector<TmxSJob>()))) {
    return rc;
  }
  if (t_total > 0 && ctx->o_npairs > 0) {
    TmxMatSet avg = {};
    avg.src[0] = (const cplx *)ctx->T.p;
    avg.dst[0] = (cplx *)ctx->Ta.p;
    tmx_launch_orient_pairs((const TmxObsGrain *)ctx->o_og.p,
                            (const int64_t *)ctx->o_pairs.p,
                            (const int32_t *)ctx->o_ord.p, ctx->o_pmax, ctx->o_npairs,
                            avg, 1, (const double *)ctx->o_coef.p, ncoef,
                            (const int64_t *)ctx->cg_off.p, (const double *)ctx->cg.p,
                            ctx->cg_nmax, ctx->o_nbmax, 0, st);
    LAUNCHED();
    std::swap(ctx->T, ctx->Ta);
  }
  CK(cudaStreamSynchronize(st));
  ctx->t_averaged = true;
  ++ctx->batch_seq;
  ctx->sink_done = 0; // the T-matrices a sink holds are the unaveraged ones
  return TMX_OK;
}

extern "C" int tmx_batch_scattering_matrix(
    tmx_ctx *ctx, int64_t njobs, const int64_t *grain, const double *alpha,
    const double *beta, const double *theta_in, const double *phi_in,
    const double *theta_out, const double *phi_out, double *Z, double *S) {
  if (!ctx || njobs < 0 || (njobs > 0 && (!grain || !alpha || !beta || !theta_in ||
                                          !phi_in || !theta_out || !phi_out ||
                                          (!Z && !S)))) {
    return TMX_ERR_INVALID;
  }
  int rc;
  if ((rc = check_jobs(ctx, njobs, grain))) {
    return rc;
  }
  CK(cudaSetDevice(ctx->device));
  std::vector<zc> SL;
  if ((rc = lab_amplitudes(ctx, njobs, grain, alpha, beta, theta_in, phi_in,
                           theta_out, phi_out, SL))) {
    return rc;
  }
  for (int64_t j = 0; j < njobs; ++j) {
    const zc M[2][2] = {{SL[4 * j], SL[4 * j + 1]}, {SL[4 * j + 2], SL[4 * j + 3]}};
    if (Z) {
      z_from_s(M, Z + 16 * j);
    }
    if (S) {
      for (int q = 0; q < 4; ++q) {
        S[8 * j + 2 * q] = SL[4 * j + q].real();
        S[8 * j + 2 * q + 1] = SL[4 * j + q].imag();
      }
    }
  }
  return TMX_OK;
}

extern "C" int tmx_batch_extinction_matrix(tmx_ctx *ctx, int64_t njobs,
                                           const int64_t *grain,
                                           const double *alpha,
                                           const double *beta,
                                           const double *theta,
                                           const double *phi, double *K) {
  if (!ctx || njobs < 0 ||
      (njobs > 0 && (!grain || !alpha || !beta || !theta || !phi || !K))) {
    return TMX_ERR_INVALID;
  }
  int rc;
  if ((rc = check_jobs(ctx, njobs, grain))) {
    return rc;
  }
  CK(cudaSetDevice(ctx->device));
  std::vector<zc> SL;
  if ((rc = lab_amplitudes(ctx, njobs, grain, alpha, beta, theta, phi, theta,
                           phi, SL))) {
    return rc;
  }
  for (int64_t j = 0; j < njobs; ++j) {
    const zc M[2][2] = {{SL[4 * j], SL[4 * j + 1]}, {SL[4 * j + 2], SL[4 * j + 3]}};
    k_from_s(ctx->up_grains[grain[j]].k, M, K + 16 * j);
  }
  return TMX_OK;
}

extern "C" int tmx_batch_absorption_cross_sections(tmx_ctx *ctx, int64_t grain,
                                                   int32_t ntheta,
                                                   const double *theta,
                                                   int32_t ngauss, double *out) {
  if (!ctx || ntheta < 0 || ngauss < 1 || (ntheta > 0 && (!theta || !out))) {
    return TMX_ERR_INVALID;
  }
  int rc;
  if ((rc = check_jobs(ctx, 1, &grain))) {
    return rc;
  }
  CK(cudaSetDevice(ctx->device));
  return absorption(ctx, (int32_t)grain, ntheta, theta, ngauss, out);
}

extern "C" int tmx_batch_average_absorption_cross_section(tmx_ctx *ctx,
                                                          int64_t grain,
                                                          int32_t ngauss,
                                                          double *out) {
  if (!ctx || ngauss < 1 || !out) {
    return TMX_ERR_INVALID;
  }
  int rc;
  if ((rc = check_jobs(ctx, 1, &grain))) {
    return rc;
  }
  CK(cudaSetDevice(ctx->device));
  // TMatrix::get_average_absorption_cross_section (TMatrix.hpp:2260-2287)
  std::vector<double> ct(ngauss), wt(ngauss), tg(ngauss), cabs(2 * ngauss);
  tmx_host_gauss_legendre(ngauss, ct.data(), wt.data());
  for (int i = 0; i < ngauss; ++i) {
    tg[i] = acos(ct[i]);
  }
  if ((rc = absorption(ctx, (int32_t)grain, ngauss, tg.data(), ngauss, cabs.data()))) {
    return rc;
  }
  double result = 0.;
  for (int i = 0; i < ngauss; ++i) {
    result += cabs[2 * i] * wt[i];
  }
  *out = 0.5 * result;
  return TMX_OK;
}
