// The plain (calculator) path: TMatrixCalculator::calculate_TMatrix
// (TMatrixCalculator.hpp:64-213) for a batch of grains on the device.
//
// Schedule, per grain (the reference runs it for one grain at a time):
//   A. nmax = int(max(4, x + 4.05 x^(1/3))), x = 2 pi R_V / lambda; while
//      nmax < maximum_order and either relative change of the m = 0 Qsca,
//      Qext exceeds the tolerance: m = 0 T-matrix at (nmax, ndgs nmax), the
//      sums over its diagonal, ++nmax; then --nmax.
//   B. ngauss = ndgs nmax + 1; while ngauss < maximum_ngauss and a change
//      exceeds the tolerance: m = 0 T-matrix at (nmax, ngauss), ++ngauss;
//      then --ngauss.
//   then every m block at (nmax, ngauss) (compute_additional_elements,
//   TMatrix.hpp:763-992).
// Every step evaluates all grains that need an m = 0 T-matrix at once: the
// table and block kernels of the batched path in chain mode (diagonal only).
// Where the reference aborts ("Unable to converge!"), the grain gets the
// TMX_GRAIN_NOT_CONVERGED bit and keeps its last order.
#include <cmath>
#include <vector>

#include "tmx_ctx.h"

namespace {

struct CalcState {
  int phase = 0; // 0: order loop, 1: quadrature loop, 2: done
  int nmax = 0, ngauss = 0;
  double old_qsca = 0., old_qext = 0.;
  double dsca = 1., dext = 1.;
};

// m = 0 class blocks of grain list `g` at orders N[i], ngauss NG[i] in chain
// mode; diag_h receives each grain's 2 N diagonal elements of T_0 (block
// index i, order n at i * N + n - 1) from diag_off[i] on.
int m0_step(tmx_ctx *ctx, const std::vector<int32_t> &g, const std::vector<int> &N,
            const std::vector<int> &NG, std::vector<cplx> &diag_h,
            std::vector<int64_t> &diag_off) {
  cudaStream_t st = ctx->stream;
  const int ns = (int)g.size();
  int rc;
  if ((rc = tmx_ensure_gl(ctx, NG))) {
    return rc;
  }
  std::vector<std::pair<int, int>> keys;
  std::map<std::pair<int, int>, int> key_idx;
  for (int s = 0; s < ns; ++s) {
    auto kk = std::make_pair(N[s], NG[s]);
    if (!key_idx.count(kk)) {
      key_idx[kk] = (int)keys.size();
      keys.push_back(kk);
    }
  }
  std::vector<int> sets;
  if ((rc = tmx_ensure_wigner(ctx, keys, false, sets))) {
    return rc;
  }
  std::vector<TmxSlot> slots(ns);
  diag_off.assign(ns, 0);
  int64_t tab = 0, nsc = 0, dg = 0;
  int ngmax = 1, nmmax = 1;
  for (int s = 0; s < ns; ++s) {
    TmxSlot &sl = slots[s];
    sl.grain = g[s];
    sl.nmax = N[s];
    sl.ngauss = NG[s];
    sl.wig_n = sets[key_idx[std::make_pair(N[s], NG[s])]];
    sl.tab = tab;
    sl.nsc = nsc;
    sl.tout = -1;
    sl.diag = dg;
    diag_off[s] = dg;
    tab += (int64_t)NG[s] * N[s] * TMX_NQ;
    nsc += (int64_t)NG[s] * TMX_NS;
    dg += 2 * (int64_t)N[s];
    ngmax = std::max(ngmax, NG[s]);
    nmmax = std::max(nmmax, N[s]);
  }
  // the four m = 0 classes of every slot, largest first
  struct It {
    int nb;
    TmxItem it;
  };
  std::vector<It> its;
  for (int s = 0; s < ns; ++s) {
    for (int c = 0; c < 4; ++c) {
      const int nb = tmx_host_class_size(N[s], 0, c);
      if (nb > 0) {
        It x;
        x.nb = nb;
        x.it.slot = s;
        x.it.m = 0;
        x.it.cls = (int16_t)c;
        x.it.scratch = 0;
        its.push_back(x);
      }
    }
  }
  std::stable_sort(its.begin(), its.end(),
                   [](const It &a, const It &b) { return a.nb > b.nb; });
  std::vector<TmxItem> items(its.size());
  int64_t scr = 0;
  for (size_t i = 0; i < its.size(); ++i) {
    items[i] = its[i].it;
    items[i].scratch = scr;
    scr += 2 * (int64_t)its[i].nb * its[i].nb;
  }
  if ((rc = ensure(ctx, ctx->tab, std::max<int64_t>(1, tab) * sizeof(double))) ||
      (rc = ensure(ctx, ctx->nsc, std::max<int64_t>(1, nsc) * sizeof(double))) ||
      (rc = ensure(ctx, ctx->scratch, std::max<int64_t>(1, scr) * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->diag, std::max<int64_t>(1, dg) * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->slots, std::max(1, ns) * sizeof(TmxSlot))) ||
      (rc = ensure(ctx, ctx->items, std::max<size_t>(1, items.size()) * sizeof(TmxItem)))) {
    return rc;
  }
  CK(cudaMemcpyAsync(ctx->slots.p, slots.data(), ns * sizeof(TmxSlot),
                     cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->items.p, items.data(), items.size() * sizeof(TmxItem),
                     cudaMemcpyHostToDevice, st));
  tmx_launch_tables((const TmxSlot *)ctx->slots.p, ns, (const TmxGrain *)ctx->grains.p,
                    (const double *)ctx->gl_x.p, (const double *)ctx->gl_w.p,
                    (const int64_t *)ctx->gl_off.p, (double *)ctx->tab.p,
                    (double *)ctx->nsc.p, ctx->up_sched.bessel_start, ngmax, nmmax, st);
  LAUNCHED();
  const int edges[] = {1 << 30, 64, 32, 16, 8, 0};
  size_t i0 = 0;
  for (int b = 0; b < 5; ++b) {
    size_t i1 = i0;
    while (i1 < its.size() && its[i1].nb > edges[b + 1]) {
      ++i1;
    }
    if (i1 > i0) {
      TmxBlockArgs B;
      B.items = (const TmxItem *)ctx->items.p + i0;
      B.nitems = (int)(i1 - i0);
      B.slots = (const TmxSlot *)ctx->slots.p;
      B.grains = (const TmxGrain *)ctx->grains.p;
      B.tab = (const double *)ctx->tab.p;
      B.nsc = (const double *)ctx->nsc.p;
      B.wig = (const double *)ctx->wig.p;
      B.wig_off = (const int64_t *)ctx->wig_off.p;
      B.scratch = (cplx *)ctx->scratch.p;
      B.tout = nullptr;
      B.diag = (cplx *)ctx->diag.p;
      B.status = (int32_t *)ctx->status.p;
      B.max_nb = its[i0].nb;
      B.chunk_nodes = tmx_host_chunk_nodes(B.max_nb);
      B.family = dispatch_family(ctx, B.max_nb);
      tmx_launch_blocks(B, st);
      LAUNCHED();
    }
    i0 = i1;
  }
  diag_h.resize(dg);
  CK(cudaMemcpyAsync(diag_h.data(), ctx->diag.p, dg * sizeof(cplx),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return TMX_OK;
}

} // namespace

extern "C" int tmx_tmatrix_batch_calculator(tmx_ctx *ctx, int64_t n,
                                            const double *r_ev,
                                            const double *wavelength,
                                            const double *mr, const double *mi,
                                            const double *axis_ratio,
                                            int32_t maximum_order,
                                            double tolerance, int32_t ndgs,
                                            int32_t maximum_ngauss) {
  if (!ctx) {
    return TMX_ERR_INVALID;
  }
  if (maximum_order < 2 || ndgs < 1 || maximum_ngauss < 1 ||
      !(tolerance >= 0.)) {
    return fail(ctx, TMX_ERR_INVALID,
                "calculator: maximum_order >= 2, ndgs >= 1, maximum_ngauss >= 1, "
                "tolerance >= 0");
  }
  // the upload keeps the grains and their input checks; of its schedule
  // only the (automatic) Bessel start rule is used here
  tmx_schedule S = {2, 3, 1, 0, tolerance};
  int rc = tmx_batch_upload(ctx, n, r_ev, wavelength, mr, mi, axis_ratio, &S);
  if (rc) {
    return rc;
  }
  CK(cudaSetDevice(ctx->device));
  NvtxRange range("tmx_calculator");
  ctx->have_batch = false;
  ctx->lu_ready = false;
  ctx->n = n;
  ++ctx->batch_seq;
  ctx->nmax_h.assign(n, 0);
  ctx->ngauss_h.assign(n, 0);
  ctx->status_h.assign(n, 0);
  ctx->q_h.assign(6 * n, 0.);
  ctx->t_off_h.assign(n, 0);
  ctx->flops_survey = 0.;
  CK(cudaMemsetAsync(ctx->status.p, 0, std::max<int64_t>(1, n) * sizeof(int32_t),
                     ctx->stream));
  std::vector<CalcState> cs(n);
  for (int64_t i = 0; i < n; ++i) {
    ctx->status_h[i] = ctx->up_status[i];
    if (ctx->up_status[i]) {
      cs[i].phase = 2;
      continue;
    }
    const double xev = 2. * M_PI * r_ev[i] / wavelength[i];
    cs[i].nmax = (int)std::max(4., xev + 4.05 * cbrt(xev));
  }
  for (;;) {
    // advance every grain to its next m = 0 evaluation (or to done)
    std::vector<int32_t> g;
    std::vector<int> N, NG;
    for (int64_t i = 0; i < n; ++i) {
      CalcState &c = cs[i];
      for (;;) {
        if (c.phase == 0) {
          if (c.nmax < maximum_order && (c.dext > tolerance || c.dsca > tolerance)) {
            break;
          }
          --c.nmax;
          if (c.nmax + 1 == maximum_order) {
            // the reference aborts; keep the last order evaluated
            ctx->status_h[i] |= TMX_GRAIN_NOT_CONVERGED;
            c.ngauss = c.nmax * ndgs;
            c.phase = 2;
            break;
          }
          c.ngauss = c.nmax * ndgs + 1;
          c.dext = tolerance + 1.;
          c.dsca = tolerance + 1.;
          c.phase = 1;
          continue;
        }
        if (c.phase == 1) {
          if (c.ngauss < maximum_ngauss && (c.dext > tolerance || c.dsca > tolerance)) {
            break;
          }
          if (c.ngauss == maximum_ngauss) {
            ctx->status_h[i] |= TMX_GRAIN_NOT_CONVERGED;
          }
          --c.ngauss;
          c.phase = 2;
        }
        break;
      }
      if (c.phase == 2) {
        continue;
      }
      const int Ni = c.nmax;
      const int NGi = (c.phase == 0) ? ndgs * c.nmax : c.ngauss;
      // the m = 0 classes of order N have at most (N + 1) / 2 members
      if (Ni < 1 || Ni > 2 * TMX_MAX_NB - 1) {
        ctx->status_h[i] |= TMX_GRAIN_TOO_LARGE;
        c.phase = 2;
        c.nmax = 0;
        continue;
      }
      g.push_back((int32_t)i);
      N.push_back(Ni);
      NG.push_back(NGi);
    }
    if (g.empty()) {
      break;
    }
    std::vector<cplx> dh;
    std::vector<int64_t> doff;
    if ((rc = m0_step(ctx, g, N, NG, dh, doff))) {
      return rc;
    }
    for (size_t s = 0; s < g.size(); ++s) {
      CalcState &c = cs[g[s]];
      const int Ni = N[s];
      const cplx *d = dh.data() + doff[s];
      // the reference's sums over T(0,n,0,0,n,0) and T(1,n,0,1,n,0)
      double qsca = 0., qext = 0.;
      for (int k = 1; k < Ni + 1; ++k) {
        const double dn1 = 2. * k + 1.;
        const cplx a = d[k - 1];
        const cplx b = d[Ni + k - 1];
        qsca += dn1 * ((a.x * a.x + a.y * a.y) + (b.x * b.x + b.y * b.y));
        qext += dn1 * (a.x + b.x);
      }
      c.dsca = std::fabs((c.old_qsca - qsca) / qsca);
      c.dext = std::fabs((c.old_qext - qext) / qext);
      c.old_qext = qext;
      c.old_qsca = qsca;
      ctx->q_h[6 * g[s] + 0] = qsca;
      ctx->q_h[6 * g[s] + 1] = qext;
      ctx->q_h[6 * g[s] + 4] = c.dsca;
      ctx->q_h[6 * g[s] + 5] = c.dext;
      if (!std::isfinite(qsca) || !std::isfinite(qext)) {
        ctx->status_h[g[s]] |= TMX_GRAIN_NAN;
        c.phase = 2;
        c.ngauss = NG[s];
      } else if (c.phase == 0) {
        ++c.nmax;
      } else {
        ++c.ngauss;
      }
    }
  }
  // every m block at the final orders; a grain whose final order has
  // classes above the block kernels' limit (in practice one that ran to
  // maximum_order without converging, where the reference aborts) gets no
  // T-matrix
  std::vector<int32_t> p2;
  std::vector<int> ngs;
  for (int64_t i = 0; i < n; ++i) {
    if (cs[i].phase == 2 && cs[i].nmax > TMX_MAX_NB) {
      ctx->status_h[i] |= TMX_GRAIN_TOO_LARGE;
      continue;
    }
    if (cs[i].phase == 2 && cs[i].nmax > 0 && cs[i].ngauss > 0 && !ctx->up_status[i]) {
      ctx->nmax_h[i] = cs[i].nmax;
      ctx->ngauss_h[i] = cs[i].ngauss;
      p2.push_back((int32_t)i);
      ngs.push_back(cs[i].ngauss);
    }
  }
  if ((rc = tmx_ensure_gl(ctx, ngs))) {
    return rc;
  }
  return tmx_run_blocks(ctx, p2);
}
