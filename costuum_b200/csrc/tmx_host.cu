// Host driver of the T-matrix library: the B200 replacement of the
// reference's TaskManager + QuickSched pair for the T-matrix path.
//
// Reference (CosTuuM): TaskManager::generate_tasks (src/TaskManager.hpp:
// 445-1346) builds, per grain, a chain InteractionTask(order) ->
// TMatrixM0Task(order) for order = min_order .. max_order - 1 that stops at
// convergence, then one TMatrixMAllTask per m; QuickSched runs the graph on
// host threads. Here the same schedule is a device work flow:
//   1. order loop ("wavefront"): every still-active grain advances one order
//      per step -- Bessel tables, the m = 0 classes (assembly + LU + solve),
//      then the convergence test and a device-side compaction of the active
//      list. The host only reads the active count between steps.
//   2. blocks: all (grain, m, class) items at the converged (nmax, ngauss),
//      bucketed by class size, largest first.
//   3. full Q sums per grain (TMatrixQTask).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "tmx_ctx.h"

// ----------------------------------------------------- Gauss-Legendre ----

// Gauss-Legendre rule of the given order on [-1, 1]: Newton iteration on
// P_n from the Lether & Wenston (1995) initial guess, ascending nodes with a
// symmetric fill. Same recipe and operation order as the reference's
// SpecialFunctions::get_gauss_legendre_points_and_weights
// (src/SpecialFunctions.hpp:646-715), so the nodes are the same doubles.
void tmx_host_gauss_legendre(int order, double *points, double *weights) {
  const unsigned ind = (unsigned)order % 2;
  const unsigned k = (unsigned)order / 2 + ind;
  for (unsigned i = 0; i < k; ++i) {
    const double theta = M_PI * (i + 0.75) / (order + 0.5);
    const double oi = 1. / order;
    const double oi2 = oi * oi;
    double x = (1. - 0.125 * oi2 + (5. / 38.) * oi * oi2 -
                (2. / 25.) * oi2 * oi2 * (1. - (14. / 39.) / (theta * theta))) *
               cos(theta);
    unsigned it = 0;
    double check = 1.e-16;
    double pa = 0., pb = 0.;
    do {
      ++it;
      if (it > 100) {
        check *= 10.;
      }
      pb = 1.;
      double pc = x;
      for (unsigned j = 1; j < (unsigned)order; ++j) {
        pa = pb;
        pb = pc;
        pc = x * pb + (x * pb - pa) * j / (j + 1.);
      }
      pa = 1. / ((pb - x * pc) * order);
      pb = pa * pc * (1. - x * x);
      x = x - pb;
    } while (fabs(pb) > check * fabs(x));
    const unsigned m = order - i - 1;
    points[m] = x;
    weights[m] = 2. * pa * pa * (1. - x * x);
    if (i != k - 1 || ind != 1) {
      points[i] = -points[m];
      weights[i] = weights[m];
    }
  }
}

static int ensure_gl(tmx_ctx *ctx, const std::vector<int> &ngs) {
  for (int ng : ngs) {
    if ((int)ctx->gl_off_h.size() <= ng) {
      ctx->gl_off_h.resize(ng + 1, -1);
    }
    if (ctx->gl_off_h[ng] >= 0) {
      continue;
    }
    std::vector<double> x(2 * ng), w(2 * ng);
    tmx_host_gauss_legendre(2 * ng, x.data(), w.data());
    ctx->gl_off_h[ng] = (int64_t)ctx->gl_x_h.size();
    ctx->gl_x_h.insert(ctx->gl_x_h.end(), x.begin(), x.begin() + ng);
    ctx->gl_w_h.insert(ctx->gl_w_h.end(), w.begin(), w.begin() + ng);
    ctx->gl_dirty = true;
  }
  if (ctx->gl_dirty) {
    int rc;
    const size_t nb = ctx->gl_x_h.size() * sizeof(double);
    if ((rc = ensure(ctx, ctx->gl_x, nb)) || (rc = ensure(ctx, ctx->gl_w, nb)) ||
        (rc = ensure(ctx, ctx->gl_off, ctx->gl_off_h.size() * sizeof(int64_t)))) {
      return rc;
    }
    CK(cudaMemcpyAsync(ctx->gl_x.p, ctx->gl_x_h.data(), nb,
                       cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->gl_w.p, ctx->gl_w_h.data(), nb,
                       cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->gl_off.p, ctx->gl_off_h.data(),
                       ctx->gl_off_h.size() * sizeof(int64_t),
                       cudaMemcpyHostToDevice, ctx->stream));
    // the host vectors must stay unchanged until the copies ran
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->gl_dirty = false;
  }
  return TMX_OK;
}

// Wigner table sets for (nmax, ngauss); all_m selects m = 0..nmax, else m = 0
static int ensure_wigner(tmx_ctx *ctx,
                         const std::vector<std::pair<int, int>> &keys,
                         bool all_m, std::vector<int> &set_ids) {
  std::vector<TmxWigJob> jobs;
  set_ids.clear();
  int max_work = 0;
  const int64_t old_used = ctx->wig_used;
  for (auto &kv : keys) {
    const auto key = std::make_tuple(kv.first, kv.second, all_m ? 1 : 0);
    auto it = ctx->wig_sets.find(key);
    if (it != ctx->wig_sets.end()) {
      set_ids.push_back(it->second);
      continue;
    }
    TmxWigJob J;
    J.nmax = kv.first;
    J.ngauss = kv.second;
    J.m_lo = 0;
    J.m_hi = all_m ? kv.first : 0;
    J.out = ctx->wig_used;
    const int64_t sz = (int64_t)(J.m_hi + 1) * J.ngauss * J.nmax * 2;
    ctx->wig_used += sz;
    const int id = (int)ctx->wig_off_h.size();
    ctx->wig_off_h.push_back(J.out);
    ctx->wig_sets[key] = id;
    set_ids.push_back(id);
    jobs.push_back(J);
    max_work = std::max(max_work, (J.m_hi + 1) * J.ngauss);
  }
  if (jobs.empty()) {
    return TMX_OK;
  }
  int rc = ensure_keep(ctx, ctx->wig, ctx->wig_used * sizeof(double),
                       old_used * sizeof(double));
  if (rc) {
    return rc;
  }
  if ((rc = ensure(ctx, ctx->wig_off, ctx->wig_off_h.size() * sizeof(int64_t)))) {
    return rc;
  }
  CK(cudaMemcpyAsync(ctx->wig_off.p, ctx->wig_off_h.data(),
                     ctx->wig_off_h.size() * sizeof(int64_t),
                     cudaMemcpyHostToDevice, ctx->stream));
  TmxWigJob *djobs = nullptr;
  CK(cudaMallocFromPoolAsync((void **)&djobs, jobs.size() * sizeof(TmxWigJob),
                             ctx->pool, ctx->stream));
  CK(cudaMemcpyAsync(djobs, jobs.data(), jobs.size() * sizeof(TmxWigJob),
                     cudaMemcpyHostToDevice, ctx->stream));
  tmx_launch_wigner(djobs, (int)jobs.size(), max_work,
                    (const double *)ctx->gl_x.p, (const int64_t *)ctx->gl_off.p,
                    (double *)ctx->wig.p, ctx->stream);
  LAUNCHED();
  CK(cudaFreeAsync(djobs, ctx->stream));
  // host vectors referenced by the async copies must outlive them
  CK(cudaStreamSynchronize(ctx->stream));
  return TMX_OK;
}

// ----------------------------------------------------------- class sizes --

// number of members of class `cls` of block m at order N (see describe() in
// tmx_blocks.cu)
static_assert(TMX_FAMILY_WARP_DFMA == TMX_BLOCKS_WARP_DFMA &&
                  TMX_FAMILY_WARP_DMMA == TMX_BLOCKS_WARP_DMMA &&
                  TMX_FAMILY_CTA32 == TMX_BLOCKS_CTA32 &&
                  TMX_FAMILY_CTA64 == TMX_BLOCKS_CTA64 &&
                  TMX_FAMILY_CTA == TMX_BLOCKS_CTA &&
                  TMX_DISPATCH_FAMILIES == TMX_BLOCK_FAMILIES,
              "public and kernel family numbers");

// largest class size of each dispatch bucket
static const int kBucketTop[TMX_DISPATCH_BUCKETS] = {8, 16, 32, 64, TMX_MAX_NB};
static const int32_t kDefaultDispatch[TMX_DISPATCH_BUCKETS] = {0, 1, 2, 3, 4};
static const char *const kFamilyNames[TMX_DISPATCH_FAMILIES] = {"warp_dfma", "warp_dmma",
                                                                "cta32", "cta64", "cta"};

int tmx_host_class_size(int N, int m, int cls) {
  if (m == 0) {
    const int n0 = (cls & 1) ? 1 : 2;
    return (N >= n0) ? (N - n0) / 2 + 1 : 0;
  }
  const int nA0 = ((m & 1) == cls) ? m : m + 1;
  const int nB0 = ((m & 1) == (cls ^ 1)) ? m : m + 1;
  const int R0 = (N >= nA0) ? (N - nA0) / 2 + 1 : 0;
  const int R1 = (N >= nB0) ? (N - nB0) / 2 + 1 : 0;
  return R0 + R1;
}

int tmx_host_chunk_nodes(int max_nb) {
  // quadrature nodes per shared-memory chunk: the assembly buffers may use
  // what the LU phase needs anyway, but at least a small floor that grows
  // with the class size (small classes keep small blocks)
  const int nrp = (max_nb + 3) / 4 * 4 + 4;
  const int ncol = (max_nb + 3) / 4 * 4;
  const size_t per_node = (size_t)(4 * nrp + 8 * ncol) * 16;
  const int lda = max_nb | 1;
  const size_t lu = ((size_t)max_nb * lda + max_nb) * 16 * 2;
  const size_t floor =
      max_nb <= 16 ? 12 * 1024 : (max_nb <= 32 ? 24 * 1024 : 64 * 1024);
  const size_t budget = std::max<size_t>(floor, std::min<size_t>(lu, 200 * 1024));
  int G = (int)(budget / per_node);
  return std::max(1, std::min(32, G));
}

extern "C" {

int64_t tmx_tmatrix_size(int32_t nmax) {
  if (nmax <= 0) {
    return 0;
  }
  int64_t s = 4 * (int64_t)nmax * nmax;
  for (int m = 1; m <= nmax; ++m) {
    const int64_t nb = nmax + 1 - m;
    s += 4 * nb * nb;
  }
  return s;
}

int tmx_create(tmx_ctx **out, int device) {
  if (!out) {
    return TMX_ERR_INVALID;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) {
    cudaGetLastError();
    return TMX_ERR_NO_DEVICE;
  }
  tmx_ctx *ctx = new tmx_ctx();
  ctx->device = device;
  int prio_lo = 0, prio_hi = 0;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) != cudaSuccess ||
      cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking,
                                   prio_hi) != cudaSuccess ||
      cudaStreamCreateWithPriority(&ctx->stream2, cudaStreamNonBlocking,
                                   prio_lo) != cudaSuccess ||
      cudaStreamCreateWithPriority(&ctx->stream3, cudaStreamNonBlocking,
                                   prio_lo) != cudaSuccess ||
      cudaStreamCreateWithPriority(&ctx->aux[0], cudaStreamNonBlocking,
                                   prio_hi) != cudaSuccess ||
      cudaStreamCreateWithPriority(&ctx->aux[1], cudaStreamNonBlocking,
                                   prio_hi) != cudaSuccess ||
      cudaStreamCreateWithPriority(&ctx->aux[2], cudaStreamNonBlocking,
                                   prio_lo) != cudaSuccess ||
      cudaStreamCreateWithPriority(&ctx->aux[3], cudaStreamNonBlocking,
                                   prio_lo) != cudaSuccess ||
      cudaStreamCreateWithPriority(&ctx->aux[4], cudaStreamNonBlocking,
                                   prio_lo) != cudaSuccess ||
      cudaStreamCreateWithPriority(&ctx->aux[5], cudaStreamNonBlocking,
                                   prio_lo) != cudaSuccess ||
      cudaMallocHost((void **)&ctx->pinned, 64) != cudaSuccess) {
    cudaGetLastError();
    for (cudaStream_t x : {ctx->stream, ctx->stream2, ctx->stream3, ctx->aux[0],
                           ctx->aux[1], ctx->aux[2], ctx->aux[3], ctx->aux[4],
                           ctx->aux[5]}) {
      if (x) {
        cudaStreamDestroy(x);
      }
    }
    delete ctx;
    return TMX_ERR_CUDA;
  }
  // a memory pool of this context: stream-ordered allocations of repeated
  // batches reuse its blocks instead of mapping new memory each time
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  // (no reuse that would make one stream wait for the other)
  uint64_t keep_all = UINT64_MAX;
  int no_deps = 0;
  if (cudaMemPoolCreate(&ctx->pool, &props) != cudaSuccess ||
      cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold,
                              &keep_all) != cudaSuccess ||
      cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolReuseAllowInternalDependencies,
                              &no_deps) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(ctx->stream);
    cudaStreamDestroy(ctx->stream2);
    cudaStreamDestroy(ctx->stream3);
    for (cudaStream_t x : ctx->aux) {
      cudaStreamDestroy(x);
    }
    cudaFreeHost(ctx->pinned);
    delete ctx;
    return TMX_ERR_CUDA;
  }
  *out = ctx;
  return TMX_OK;
}

void tmx_destroy(tmx_ctx *ctx) {
  if (!ctx) {
    return;
  }
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->stream2) {
    cudaStreamSynchronize(ctx->stream2);
  }
  if (ctx->stream3) {
    cudaStreamSynchronize(ctx->stream3);
  }
  for (cudaStream_t x : ctx->aux) {
    if (x) {
      cudaStreamSynchronize(x);
    }
  }
  if (ctx->t0) {
    cudaEventDestroy(ctx->t0);
    cudaEventDestroy(ctx->t1);
  }
  for (cudaEvent_t e : ctx->prof_pool) {
    cudaEventDestroy(e);
  }
  if (ctx->tl_origin) {
    cudaEventDestroy(ctx->tl_origin);
  }
  for (cudaEvent_t e : ctx->drain_ev) {
    if (e) {
      cudaEventDestroy(e);
    }
  }
  if (ctx->gm_exec) {
    cudaGraphExecDestroy(ctx->gm_exec);
  }
  if (ctx->gm_graph) {
    cudaGraphDestroy(ctx->gm_graph);
  }
  DevBuf *gm_bufs[] = {&ctx->gm_state, &ctx->gm_iter, &ctx->gm_tab, &ctx->gm_nsc,
                       &ctx->gm_scr, &ctx->gm_diag, &ctx->gm_slots, &ctx->gm_items,
                       &ctx->gm_rslots, &ctx->gm_bitems, &ctx->gm_bptr, &ctx->gm_bcap,
                       &ctx->gm_tpl, &ctx->gm_tpl_off, &ctx->gm_full,
                       &ctx->gm_tsize, &ctx->gm_toff, &ctx->gm_lu, &ctx->gm_luscr,
                       &ctx->gm_allitems, &ctx->gm_steps};
  for (DevBuf *b : gm_bufs) {
    if (b->p) {
      cudaFreeAsync(b->p, ctx->stream);
    }
  }
  for (cudaStream_t x : {ctx->gm_cs, ctx->gm_rs}) {
    if (x) {
      cudaStreamDestroy(x);
    }
  }
  for (cudaStream_t x : ctx->gm_bs) {
    if (x) {
      cudaStreamDestroy(x);
    }
  }
  DevBuf *bufs[] = {&ctx->lu, &ctx->dT, &ctx->tscr, &ctx->dTa, &ctx->dS,
                    &ctx->cg, &ctx->cg_off, &ctx->Ta, &ctx->o_angles,
                    &ctx->o_phis, &ctx->o_wts, &ctx->o_coef, &ctx->o_shw,
                    &ctx->o_og, &ctx->o_work, &ctx->o_sj, &ctx->o_qj, &ctx->o_S,
                    &ctx->o_gq, &ctx->o_gz, &ctx->o_cq, &ctx->o_cz,
                    &ctx->o_pairs, &ctx->o_grp, &ctx->o_x, &ctx->o_ord, &ctx->o_wcol,
                    &ctx->p2tab, &ctx->p2nsc, &ctx->p2scratch, &ctx->p2slots,
                    &ctx->p2items, &ctx->done, &ctx->keep_arena, &ctx->keep_tab,
                    &ctx->keep_q, &ctx->done_pos, &ctx->keep_ctl,
                    &ctx->state0, &ctx->actinit,
                    &ctx->gl_x,  &ctx->gl_w,   &ctx->gl_off,  &ctx->wig,
                    &ctx->wig_off, &ctx->grains, &ctx->state,  &ctx->act0,
                    &ctx->act1,  &ctx->count,  &ctx->slots,   &ctx->items,
                    &ctx->tab,   &ctx->nsc,    &ctx->scratch, &ctx->diag,
                    &ctx->T,     &ctx->q,
                    &ctx->status, &ctx->probe};
  for (DevBuf *b : bufs) {
    if (b->p) {
      cudaFreeAsync(b->p, ctx->stream);
    }
  }
  cudaStreamSynchronize(ctx->stream);
  if (ctx->pinned_done) {
    cudaFreeHost(ctx->pinned_done);
  }
  if (ctx->pinned_keep) {
    cudaFreeHost(ctx->pinned_keep);
  }
  if (ctx->pinned) {
    cudaFreeHost(ctx->pinned);
  }
  cudaStreamDestroy(ctx->stream);
  if (ctx->stream2) {
    cudaStreamDestroy(ctx->stream2);
  }
  if (ctx->stream3) {
    cudaStreamDestroy(ctx->stream3);
  }
  for (cudaStream_t x : ctx->aux) {
    if (x) {
      cudaStreamDestroy(x);
    }
  }
  if (ctx->copy_stream) {
    cudaStreamDestroy(ctx->copy_stream);
  }
  if (ctx->pool) {
    cudaMemPoolDestroy(ctx->pool);
  }
  delete ctx;
}

const char *tmx_last_error(const tmx_ctx *ctx) {
  return ctx ? ctx->err.c_str() : "no context";
}

int64_t tmx_kernel_launches(const tmx_ctx *ctx) {
  return ctx ? ctx->launches : 0;
}

int tmx_batch_upload(tmx_ctx *ctx, int64_t n, const double *r_ev,
                     const double *wavelength, const double *mr,
                     const double *mi, const double *axis_ratio,
                     const tmx_schedule *sched) {
  if (!ctx) {
    return TMX_ERR_INVALID;
  }
  if (n < 0 || (n > 0 && (!r_ev || !wavelength || !mr || !mi || !axis_ratio))) {
    return fail(ctx, TMX_ERR_INVALID, "null input array or negative n");
  }
  tmx_schedule S = {10, 100, 2, 0, 1.e-4};
  if (sched) {
    S = *sched;
  }
  if (S.bessel_start < 0) {
    S.bessel_start = 0;
  }
  if (S.min_order < 2 || S.max_order <= S.min_order ||
      S.gauss_legendre_factor < 1 || !(S.tolerance >= 0.)) {
    return fail(ctx, TMX_ERR_INVALID,
                "schedule needs 2 <= min_order < max_order, factor >= 1, "
                "tolerance >= 0");
  }
  if (S.max_order - 1 > TMX_MAX_NB) {
    return fail(ctx, TMX_ERR_INVALID,
                "max_order - 1 exceeds the on-chip block limit " +
                    std::to_string(TMX_MAX_NB));
  }
  if (S.bessel_start > 0 && (S.bessel_start < S.max_order || S.bessel_start > 800)) {
    return fail(ctx, TMX_ERR_INVALID,
                "bessel_start must be 0 (automatic) or in [max_order, 800]");
  }
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  ctx->uploaded = false;
  ctx->keep_valid = false;
  ctx->have_batch = false;
  int rc;
  if ((rc = tmx_release_rounds(ctx))) {
    return rc;
  }

  // ---- grains (host constants, as the reference computes them)
  std::vector<TmxGrain> gr(n);
  std::vector<int32_t> act;
  act.reserve(n);
  std::vector<TmxChainState> st0(n);
  for (int64_t i = 0; i < n; ++i) {
    TmxGrain &g = gr[i];
    g.r_ev = r_ev[i];
    g.k = 2. * M_PI / wavelength[i];
    g.mr = mr[i];
    g.mi = mi[i];
    g.axis_ratio = axis_ratio[i];
    g.cbrt_d = cbrt(axis_ratio[i]);
    TmxChainState &s = st0[i];
    s.qsca = s.qext = 0.;
    s.dqs_t = s.dqe_t = -2.;
    s.dqs = s.dqe = -1.;
    s.nmax = s.ngauss = 0;
    s.converged = 0;
    s.status = 0;
    const bool ok = std::isfinite(r_ev[i]) && r_ev[i] > 0. &&
                    std::isfinite(wavelength[i]) && wavelength[i] > 0. &&
                    std::isfinite(axis_ratio[i]) && axis_ratio[i] > 0. &&
                    std::isfinite(mr[i]) && std::isfinite(mi[i]);
    if (ok) {
      act.push_back((int32_t)i);
    } else {
      s.status = TMX_ST_BAD_INPUT;
    }
  }
  if ((rc = ensure(ctx, ctx->grains, n * sizeof(TmxGrain))) ||
      (rc = ensure(ctx, ctx->state, n * sizeof(TmxChainState))) ||
      (rc = ensure(ctx, ctx->state0, n * sizeof(TmxChainState))) ||
      (rc = ensure(ctx, ctx->actinit, n * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->act0, n * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->act1, n * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->count, 16)) ||
      (rc = ensure(ctx, ctx->status, n * sizeof(int32_t)))) {
    return rc;
  }
  CK(cudaMemcpyAsync(ctx->grains.p, gr.data(), n * sizeof(TmxGrain),
                     cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->state0.p, st0.data(), n * sizeof(TmxChainState),
                     cudaMemcpyHostToDevice, st));
  if (!act.empty()) {
    CK(cudaMemcpyAsync(ctx->actinit.p, act.data(), act.size() * sizeof(int32_t),
                       cudaMemcpyHostToDevice, st));
  }
  // the host arrays above are about to go out of scope
  CK(cudaStreamSynchronize(st));
  ++ctx->batch_seq;
  ctx->up_n = n;
  ctx->up_grains = gr;
  ctx->up_nact = (int)act.size();
  ctx->up_sched = S;
  ctx->up_status.resize(n);
  for (int64_t i = 0; i < n; ++i) {
    ctx->up_status[i] = st0[i].status;
  }
  ctx->uploaded = true;
  return TMX_OK;
}

// One round of phase 2: every (grain, m, class) block of the grains in p2 at
// their orders (ctx->nmax_h / ctx->ngauss_h), launched on stream `st`, with
// T-matrices from complex offset t_base on (keep_T: T already holds earlier
// rounds below t_base). The schedule is kept in the context (p2 buffers and
// ctx->p2_*) for the tangent kernels. Host-side setup runs on ctx->stream
// (Wigner tables), which the round then waits for.
static int run_blocks_round(tmx_ctx *ctx, const std::vector<int32_t> &p2,
                            cudaStream_t st, int64_t t_base, bool keep_T,
                            int64_t *t_end, bool temp = false,
                            bool keep_lu = false) {
  int rc;
  NvtxRange blocks_range("tmx_blocks");
  const int np2 = (int)p2.size();
  const int64_t wig_used0 = ctx->wig_used;
  const void *T_before = ctx->T.p, *q_before = ctx->q.p;
  if (!keep_T) {
    ctx->sink_done = 0; // a new set of T-matrices starts at offset 0
  }
  std::vector<TmxSlot> slots(np2);
  std::vector<std::pair<int, int>> keys;
  std::map<std::pair<int, int>, int> key_idx;
  int64_t tab_total = 0, nsc_total = 0, t_total = t_base;
  for (int s = 0; s < np2; ++s) {
    const int g = p2[s];
    const int N = ctx->nmax_h[g], ng = ctx->ngauss_h[g];
    auto kk = std::make_pair(N, ng);
    if (!key_idx.count(kk)) {
      key_idx[kk] = (int)keys.size();
      keys.push_back(kk);
    }
    TmxSlot &sl = slots[s];
    sl.grain = g;
    sl.nmax = N;
    sl.ngauss = ng;
    sl.tab = tab_total;
    sl.nsc = nsc_total;
    sl.tout = t_total;
    sl.diag = 0;
    ctx->t_off_h[g] = t_total;
    tab_total += (int64_t)ng * N * TMX_NQ;
    nsc_total += (int64_t)ng * TMX_NS;
    t_total += tmx_tmatrix_size(N);
  }
  *t_end = t_total;
  // A round of the order loop takes its grains' final-order tables from
  // the batch's arena, where the loop copied them (k_keep_tables), instead
  // of computing them again -- if every grain of the round has a copy.
  bool kept = temp && ctx->keep_valid && np2 > 0;
  for (int s = 0; kept && s < np2; ++s) {
    kept = ctx->keep_off_h[p2[s]] >= 0;
  }
  if (kept) {
    for (int s = 0; s < np2; ++s) {
      TmxSlot &sl = slots[s];
      sl.tab = ctx->keep_off_h[sl.grain];
      // (k_keep_tables puts the node scalars at the next multiple of 16)
      sl.nsc = sl.tab + (((int64_t)sl.ngauss * sl.nmax * TMX_NQ + 15) & ~(int64_t)15);
    }
  }
  std::vector<int> full_sets;
  if ((rc = ensure_wigner(ctx, keys, true, full_sets))) {
    return rc;
  }
  for (int s = 0; s < np2; ++s) {
    slots[s].wig_n = full_sets[key_idx[std::make_pair(slots[s].nmax, slots[s].ngauss)]];
  }
  // items, ordered by class size (largest first; a counting sort, stable in
  // (slot, m, class) order), from a per-order template of a grain's items
  for (int s = 0; s < np2; ++s) {
    const int N = slots[s].nmax;
    if ((int)ctx->item_tpl.size() <= N) {
      ctx->item_tpl.resize(N + 1);
    }
    tmx_ctx::ItemTemplate &tp = ctx->item_tpl[N];
    if (tp.mc.empty() && N > 0) {
      std::vector<int32_t> c(TMX_MAX_NB + 2, 0);
      for (int m = 0; m <= N; ++m) {
        const int ncls = (m == 0) ? 4 : 2;
        for (int cl = 0; cl < ncls; ++cl) {
          const int nb = tmx_host_class_size(N, m, cl);
          if (nb > 0) {
            tp.mc.push_back((m << 8) | cl);
            tp.nb.push_back(nb);
            c[std::min(nb, TMX_MAX_NB + 1)] += 1;
            tp.fl_a += item_flops(nb, m, 1) - item_flops(nb, m, 0);
            tp.fl_b += item_flops(nb, m, 0);
          }
        }
      }
      for (int b = 0; b < TMX_MAX_NB + 2; ++b) {
        if (c[b]) {
          tp.bins.push_back(std::make_pair(b, c[b]));
        }
      }
    }
  }
  std::vector<int64_t> cnt(TMX_MAX_NB + 2, 0);
  int64_t nitems = 0;
  for (int s = 0; s < np2; ++s) {
    for (const auto &bc : ctx->item_tpl[slots[s].nmax].bins) {
      cnt[bc.first] += bc.second;
      nitems += bc.second;
    }
  }
  std::vector<int64_t> pos(TMX_MAX_NB + 2, 0);
  for (int nb = TMX_MAX_NB + 1, acc = 0; nb >= 1; --nb) {
    pos[nb] = acc;
    acc += (int)cnt[nb];
  }
  std::vector<TmxItem> &items = ctx->p2_items;
  std::vector<int> &inb = ctx->p2_nb;
  items.resize(nitems);
  inb.resize(nitems);
  for (int s = 0; s < np2; ++s) {
    const tmx_ctx::ItemTemplate &tp = ctx->item_tpl[slots[s].nmax];
    const int ni = (int)tp.mc.size();
    for (int j = 0; j < ni; ++j) {
      const int nb = tp.nb[j];
      const int64_t i = pos[std::min(nb, TMX_MAX_NB + 1)]++;
      TmxItem &it = items[i];
      it.slot = s;
      it.m = (int16_t)(tp.mc[j] >> 8);
      it.cls = (int16_t)(tp.mc[j] & 0xff);
      inb[i] = nb;
    }
  }
  ctx->p2_slots = slots;
  int64_t scr_total = 0;
  for (int64_t i = 0; i < nitems; ++i) {
    items[i].scratch = scr_total;
    scr_total += 2 * (int64_t)inb[i] * inb[i];
  }
  ctx->p2_scr_total = scr_total;
  if (keep_T && (size_t)t_total * sizeof(cplx) > ctx->T.cap) {
    // growing T moves it: earlier rounds on the round streams must be done
    CK(cudaStreamSynchronize(ctx->stream2));
    CK(cudaStreamSynchronize(ctx->stream3));
  }
  if ((rc = (keep_T ? ensure_keep(ctx, ctx->T, std::max<int64_t>(1, t_total) * sizeof(cplx),
                                  t_base * sizeof(cplx))
                    : ensure(ctx, ctx->T, std::max<int64_t>(1, t_total) * sizeof(cplx))))) {
    return rc;
  }
  if (!temp &&
      ((rc = ensure(ctx, ctx->p2tab, std::max<int64_t>(1, tab_total) * sizeof(double))) ||
       (rc = ensure(ctx, ctx->p2nsc, std::max<int64_t>(1, nsc_total) * sizeof(double))) ||
       (rc = ensure(ctx, ctx->p2scratch, std::max<int64_t>(1, scr_total) * sizeof(cplx))) ||
       (rc = ensure(ctx, ctx->p2slots, std::max(1, np2) * sizeof(TmxSlot))) ||
       (rc = ensure(ctx, ctx->p2items, std::max<int64_t>(1, nitems) * sizeof(TmxItem))))) {
    return rc;
  }
  // a single round on persistent buffers can keep the LU factors of every
  // item for a later gradient pass (same item order and scratch offsets)
  if (keep_lu &&
      (rc = ensure(ctx, ctx->lu, std::max<int64_t>(1, scr_total) * sizeof(cplx)))) {
    return rc;
  }
  if (ctx->q.cap < (size_t)2 * ctx->n * sizeof(double)) {
    // Q sums of every grain of the batch; rounds on the round streams may
    // still write the old buffer
    CK(cudaStreamSynchronize(ctx->stream2));
    CK(cudaStreamSynchronize(ctx->stream3));
    if ((rc = ensure(ctx, ctx->q, std::max<int64_t>(1, 2 * ctx->n) * sizeof(double)))) {
      return rc;
    }
  }
  if (np2 == 0) {
    return TMX_OK;
  }
  if (st != ctx->stream && (!temp || ctx->wig_used != wig_used0 ||
                            ctx->T.p != T_before || ctx->q.p != q_before)) {
    // new Wigner tables or a moved T / Q-sum buffer above are ordered on
    // ctx->stream (a round of the order loop that needs none of them does
    // not wait for the orders queued there)
    cudaEvent_t ready;
    CK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    CK(cudaEventRecord(ready, ctx->stream));
    CK(cudaStreamWaitEvent(st, ready, 0));
    CK(cudaEventDestroy(ready));
  }
  // buffers of this round: the persistent p2 set, or (temp) stream-ordered
  // allocations on `st` that are released after the round's launches
  double *tab = (double *)ctx->p2tab.p, *nsc = (double *)ctx->p2nsc.p;
  cplx *scratch = (cplx *)ctx->p2scratch.p;
  TmxSlot *dslots = (TmxSlot *)ctx->p2slots.p;
  TmxItem *ditems = (TmxItem *)ctx->p2items.p;
  if (kept) {
    tab = nsc = (double *)ctx->keep_arena.p;
  } else if (temp) {
    CK(cudaMallocFromPoolAsync((void **)&tab, std::max<int64_t>(1, tab_total) * sizeof(double), ctx->pool, st));
    CK(cudaMallocFromPoolAsync((void **)&nsc, std::max<int64_t>(1, nsc_total) * sizeof(double), ctx->pool, st));
  }
  if (temp) {
    CK(cudaMallocFromPoolAsync((void **)&scratch, std::max<int64_t>(1, scr_total) * sizeof(cplx), ctx->pool, st));
    CK(cudaMallocFromPoolAsync((void **)&dslots, np2 * sizeof(TmxSlot), ctx->pool, st));
    CK(cudaMallocFromPoolAsync((void **)&ditems, std::max<int64_t>(1, nitems) * sizeof(TmxItem), ctx->pool, st));
  }
  // a kept round also keeps its items' LU factors for the gradients
  cplx *lu_keep = nullptr;
  if (temp && ctx->keep_rounds) {
    CK(cudaMallocFromPoolAsync((void **)&lu_keep, std::max<int64_t>(1, scr_total) * sizeof(cplx),
                               ctx->pool, st));
  }
  CK(cudaMemcpyAsync(dslots, slots.data(), np2 * sizeof(TmxSlot),
                     cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ditems, items.data(), nitems * sizeof(TmxItem),
                     cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync((cplx *)ctx->T.p + t_base, 0, (t_total - t_base) * sizeof(cplx), st));
  cudaEvent_t pe = nullptr;
  if (!kept) {
    if ((rc = prof_begin(ctx, 1, &pe, st))) {
      return rc;
    }
    int ngmax = 1, nmmax = 1;
    for (const TmxSlot &sl : slots) {
      ngmax = std::max(ngmax, sl.ngauss);
      nmmax = std::max(nmmax, sl.nmax);
    }
    tmx_launch_tables(dslots, np2, (const TmxGrain *)ctx->grains.p,
                      (const double *)ctx->gl_x.p, (const double *)ctx->gl_w.p,
                      (const int64_t *)ctx->gl_off.p, tab, nsc,
                      ctx->up_sched.bessel_start, ngmax, nmmax, st);
    LAUNCHED();
    if ((rc = prof_end(ctx, 1, pe, 0., st, 0., np2))) {
      return rc;
    }
  }
  // class-size buckets, one launch each (largest first): the first on `st`,
  // the others on the two auxiliary streams beside it, so that the smaller
  // buckets fill the SMs that the tail of the larger one leaves idle; the
  // round ends (Q sums, buffer release) when all of them are done
  cudaStream_t *aux = (st == ctx->stream)    ? &ctx->aux[0]
                      : (st == ctx->stream2) ? &ctx->aux[2]
                                             : &ctx->aux[4];
  // the point on `st` (tables and lists ready) after which every bucket may
  // start: recorded before the first bucket's launch, so that the others
  // run beside it rather than after it
  cudaEvent_t fork = nullptr;
  if (!ctx->tuning && nitems > 0 &&
      dispatch_bucket(inb[0]) != dispatch_bucket(inb[nitems - 1])) {
    CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    CK(cudaEventRecord(fork, st));
  }
  std::vector<cudaEvent_t> joins;
  int nbuckets = 0;
  const int edges[] = {1 << 30, 64, 32, 16, 8, 0};
  int64_t i0 = 0;
  for (int b = 0; b < 5; ++b) {
    int64_t i1 = i0;
    while (i1 < nitems && inb[i1] > edges[b + 1]) {
      ++i1;
    }
    if (i1 > i0) {
      cudaStream_t bs = st;
      // while tuning, every bucket runs alone on the round's stream
      if (nbuckets > 0 && !ctx->tuning) {
        bs = aux[(nbuckets - 1) & 1];
        CK(cudaStreamWaitEvent(bs, fork, 0));
      }
      ++nbuckets;
      TmxBlockArgs B;
      B.items = ditems + i0;
      B.nitems = (int)(i1 - i0);
      B.slots = dslots;
      B.grains = (const TmxGrain *)ctx->grains.p;
      B.tab = tab;
      B.nsc = nsc;
      B.wig = (const double *)ctx->wig.p;
      B.wig_off = (const int64_t *)ctx->wig_off.p;
      B.scratch = scratch;
      B.tout = (cplx *)ctx->T.p;
      B.diag = nullptr;
      B.status = (int32_t *)ctx->status.p;
      B.max_nb = inb[i0];
      B.chunk_nodes = tmx_host_chunk_nodes(B.max_nb);
      B.lu = keep_lu ? (cplx *)ctx->lu.p : lu_keep;
      B.family = dispatch_family(ctx, B.max_nb);
      // the round's flops are booked on its first launch
      double fl = 0.;
      if (ctx->profiling && nbuckets == 1) {
        for (int s = 0; s < np2; ++s) {
          const tmx_ctx::ItemTemplate &tp = ctx->item_tpl[slots[s].nmax];
          fl += tp.fl_a * slots[s].ngauss + tp.fl_b;
        }
      }
      if ((rc = prof_begin(ctx, 0, &pe, bs))) {
        return rc;
      }
      cudaEvent_t ta = nullptr, tb = nullptr;
      if (ctx->tuning) {
        CK(cudaEventCreate(&ta));
        CK(cudaEventCreate(&tb));
        CK(cudaEventRecord(ta, bs));
      }
      tmx_launch_blocks(B, bs);
      LAUNCHED();
      if (ctx->tuning) {
        CK(cudaEventRecord(tb, bs));
        ctx->tune_ev.emplace_back(dispatch_bucket(B.max_nb), ta, tb);
      }
      if ((rc = prof_end(ctx, 0, pe, fl, bs, 0., B.nitems))) {
        return rc;
      }
      if (bs != st) {
        cudaEvent_t j;
        CK(cudaEventCreateWithFlags(&j, cudaEventDisableTiming));
        CK(cudaEventRecord(j, bs));
        joins.push_back(j);
      }
    }
    i0 = i1;
  }
  for (cudaEvent_t j : joins) {
    CK(cudaStreamWaitEvent(st, j, 0));
    CK(cudaEventDestroy(j));
  }
  if (fork) {
    CK(cudaEventDestroy(fork));
  }
  tmx_launch_qsums(dslots, np2, (const cplx *)ctx->T.p, (double *)ctx->q.p, st);
  LAUNCHED();
  // the round's T-matrices to the caller's page-locked sink, on the copy
  // stream once the round is done: the copy overlaps the order loop and the
  // rounds that follow, which do not wait for it (the batch's end does)
  if (ctx->sink && t_base == ctx->sink_done && t_total <= ctx->sink_cap &&
      t_total > t_base) {
    if (!ctx->copy_stream) {
      CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    }
    cudaEvent_t done;
    CK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    CK(cudaEventRecord(done, st));
    CK(cudaStreamWaitEvent(ctx->copy_stream, done, 0));
    CK(cudaEventDestroy(done));
    CK(cudaMemcpyAsync(ctx->sink + 2 * t_base, (const cplx *)ctx->T.p + t_base,
                       (t_total - t_base) * sizeof(cplx), cudaMemcpyDeviceToHost,
                       ctx->copy_stream));
    ctx->sink_done = t_total;
    if (st == ctx->stream) {
      // a round on the library stream ends its batch (a single round, or
      // the last one): the batch's synchronisation covers the copy
      CK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
      CK(cudaEventRecord(done, ctx->copy_stream));
      CK(cudaStreamWaitEvent(st, done, 0));
      CK(cudaEventDestroy(done));
    }
  }
  if (temp && ctx->keep_rounds) {
    tmx_ctx::RoundRec rec;
    rec.tab = tab;
    rec.nsc = nsc;
    rec.own_tables = !kept;
    rec.slots = dslots;
    rec.items = ditems;
    rec.lu = lu_keep;
    rec.nb = inb;
    rec.scr_total = scr_total;
    ctx->rounds_kept.push_back(std::move(rec));
    CK(cudaFreeAsync(scratch, st));
  } else if (temp) {
    if (!kept) {
      CK(cudaFreeAsync(tab, st));
      CK(cudaFreeAsync(nsc, st));
    }
    CK(cudaFreeAsync(scratch, st));
    CK(cudaFreeAsync(dslots, st));
    CK(cudaFreeAsync(ditems, st));
  }
  return TMX_OK;
}

// End of a batch: full Q sums of every grain (TMatrixQTask) on ctx->stream
// after all block rounds, per-grain results to the host.
// (q2_in, stb_in: the Q sums and status words already read back, if given)
static int finish_blocks(tmx_ctx *ctx, int64_t t_total, int rounds,
                         const std::vector<double> *q2_in = nullptr,
                         const std::vector<int32_t> *stb_in = nullptr) {
  cudaStream_t st = ctx->stream;
  const int64_t n = ctx->n;
  const tmx_schedule S = ctx->up_sched;
  const int glf = S.gauss_legendre_factor;
  int rc;
  ctx->p2_t_total = t_total;
  ctx->p2_rounds = rounds;
  ctx->t_averaged = false;
  ++ctx->batch_seq;
  if (t_total > 0) {
    std::vector<double> q2;
    std::vector<int32_t> stb;
    if (q2_in && stb_in) {
      q2 = *q2_in;
      stb = *stb_in;
    } else {
      q2.resize(2 * n);
      stb.resize(n);
      CK(cudaMemcpyAsync(q2.data(), ctx->q.p, 2 * n * sizeof(double),
                         cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(stb.data(), ctx->status.p, n * sizeof(int32_t),
                         cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    }
    for (int64_t i = 0; i < n; ++i) {
      if (ctx->nmax_h[i] > 0) {
        ctx->q_h[6 * i + 2] = q2[2 * i];
        ctx->q_h[6 * i + 3] = q2[2 * i + 1];
      }
      ctx->status_h[i] |= stb[i];
    }
  }
  // survey-model flops (per grain: every order of the m = 0 chain on the
  // unreduced 2k x 2k block, then every m >= 1 block on 2nm x 2nm)
  // (cumulative per-order sums, cached for this glf and minimum order):
  // grain flops = chain[N] + ng * mg[N] + mc[N]
  std::vector<double> &sc = ctx->survey_cache;
  if (ctx->profiling && (ctx->survey_glf != glf || ctx->survey_min != S.min_order)) {
    sc.clear();
    ctx->survey_glf = glf;
    ctx->survey_min = S.min_order;
  }
  for (int64_t i = 0; ctx->profiling && i < n; ++i) {
    const int N = ctx->nmax_h[i];
    if (N <= 0) {
      continue;
    }
    for (int k = (int)(sc.size() / 3); k <= N; ++k) {
      const double b = k, g = glf * k, t = 2. * k;
      double chain = k ? sc[3 * (k - 1)] : 0., mg = k ? sc[3 * k - 2] : 0.,
             mc = k ? sc[3 * k - 1] : 0.;
      if (k >= S.min_order) {
        chain += 8. * 4. * b * b * g + (8. / 3.) * t * t * t + 8. * t * t * t;
      }
      if (k >= 1) { // the m >= 1 block of size b = k
        mg += 8. * 10. * b * b;
        mc += (8. / 3.) * t * t * t + 8. * t * t * t;
      }
      sc.push_back(chain);
      sc.push_back(mg);
      sc.push_back(mc);
    }
    ctx->flops_survey += sc[3 * N] + ctx->ngauss_h[i] * sc[3 * N + 1] + sc[3 * N + 2];
  }
  // event pairs are resolved when the profile is read; a long profiled run
  // resolves here now and then so that the pool stays bounded
  if (ctx->prof_used > 8192 && (rc = prof_resolve(ctx))) {
    return rc;
  }
  ctx->have_batch = true;
  return TMX_OK;
}

// Buffers of the kept rounds of the previous batch back to the pool (that
// batch has finished: every batch ends with a host synchronisation).
int tmx_release_rounds(tmx_ctx *ctx) {
  for (auto &r : ctx->rounds_kept) {
    if (!r.own_tables) {
      r.tab = r.nsc = nullptr; // the batch's table arena
    }
    if (r.borrowed) {
      r.slots = nullptr;
      r.items = nullptr;
      r.lu = nullptr;
    }
    for (void *p : {(void *)r.tab, (void *)r.nsc, (void *)r.slots, (void *)r.items,
                    (void *)r.lu}) {
      if (p) {
        CK(cudaFreeAsync(p, ctx->stream));
      }
    }
  }
  ctx->rounds_kept.clear();
  ctx->rounds_lu = false;
  return TMX_OK;
}

// Phase 2 in one round for the grains in p2 (all grains with an order).
static int run_blocks(tmx_ctx *ctx, const std::vector<int32_t> &p2) {
  int64_t t_end = 0;
  int rc = run_blocks_round(ctx, p2, ctx->stream, 0, false, &t_end, false, true);
  if (rc) {
    return rc;
  }
  ctx->lu_ready = true;
  return finish_blocks(ctx, t_end, 1);
}

// Phase 2 again in one round for the last batch, so that the p2 buffers hold
// the whole schedule (after a batch whose blocks ran in two rounds).
int tmx_rerun_blocks(tmx_ctx *ctx) {
  std::vector<int32_t> p2;
  for (int64_t i = 0; i < ctx->n; ++i) {
    if (ctx->nmax_h[i] > 0) {
      p2.push_back((int32_t)i);
    }
  }
  int64_t t_end = 0;
  // the same T-matrices again: what the sink holds stays valid
  double *sink = ctx->sink;
  const int64_t sink_done = ctx->sink_done;
  ctx->sink = nullptr;
  int rc = run_blocks_round(ctx, p2, ctx->stream, 0, false, &t_end, false, true);
  ctx->sink = sink;
  ctx->sink_done = sink_done;
  if (rc) {
    return rc;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->p2_t_total = t_end;
  ctx->p2_rounds = 1;
  ctx->lu_ready = true;
  return TMX_OK;
}


// ------------------------------------------------- device-driven batch --
//
// tmx_batch_compute in TMX_BATCH_GRAPH mode: the kernels of tmx_graph.cu and
// the existing step kernels captured once per batch shape into a CUDA graph
// whose WHILE node runs the order loop and its rounds on the device.
// Returns TMX_OK, an error, or 1 when this batch must run in the host mode
// (not covered, or the T-matrix / LU storage ran out: the hints grow).

// most CTAs of a round's block launch (the items of a round are known only
// on the device; each CTA loops over its share)
#ifndef TMX_GM_ROUND_CTAS
#define TMX_GM_ROUND_CTAS (148 * 16)
#endif

// largest final order of the batch just computed, for the extent of the
// next device-driven graph of the same schedule
static void note_kmax(tmx_ctx *ctx) {
  int km = 0;
  for (int32_t v : ctx->nmax_h) {
    km = std::max(km, (int)v);
  }
  ctx->kmax_seen = km;
  ctx->kmax_sched[0] = ctx->up_sched.min_order;
  ctx->kmax_sched[1] = ctx->up_sched.max_order - 1;
  ctx->kmax_sched[2] = ctx->up_sched.gauss_legendre_factor;
  ctx->kmax_tol = ctx->up_sched.tolerance;
}

static int gm_bucket(int nb) {
  return (nb <= 8) ? 0 : (nb <= 16) ? 1 : (nb <= 32) ? 2 : (nb <= 64) ? 3 : 4;
}

static int gm_compute(tmx_ctx *ctx) {
  cudaStream_t st = ctx->stream;
  const int64_t n = ctx->up_n;
  const tmx_schedule S = ctx->up_sched;
  const int glf = S.gauss_legendre_factor;
  const int K = S.max_order - 1;
  const int kmin = S.min_order;
  int rc;
  if (ctx->up_nact <= 0 || n > (1 << 22) || K < kmin || K > 100 || ctx->profiling ||
      ctx->tuning) {
    return 1;
  }
  // The graph's orders end 8 above the largest final order of the previous
  // batch of the same schedule (the orders beyond it would only be skipped
  // nodes at the ends of both chains); a batch with grains still active at
  // that order runs again in the host-driven mode, whose orders then set the
  // bound of the next graph. Convergence still uses the schedule's last order.
  // The order steps' tables and the arena of final-order tables are sized
  // for orders up to Kg.
  // (The extent only grows while the schedule stays the same, so that
  // batches of changing orders -- one grain per call, say -- reuse one graph
  // instead of building one per extent.)
  int Kg = K;
  if (ctx->kmax_seen > 0 && ctx->kmax_sched[0] == kmin && ctx->kmax_sched[1] == K &&
      ctx->kmax_sched[2] == glf && ctx->kmax_tol == S.tolerance) {
    Kg = std::min(K, std::max(kmin, ctx->kmax_seen + 8));
    if (ctx->gm_kg > 0 && ctx->gm_kg_sched[0] == kmin && ctx->gm_kg_sched[1] == K &&
        ctx->gm_kg_sched[2] == glf && ctx->gm_kg_tol == S.tolerance) {
      Kg = std::max(Kg, ctx->gm_kg);
    }
  }
  ctx->gm_kg = Kg;
  ctx->gm_kg_sched[0] = kmin;
  ctx->gm_kg_sched[1] = K;
  ctx->gm_kg_sched[2] = glf;
  ctx->gm_kg_tol = S.tolerance;
  const double tab_per = (double)glf * Kg * Kg * TMX_NQ + (double)glf * Kg * TMX_NS + 32.;
  if (2. * tab_per * sizeof(double) * n > 24e9) {
    return 1;
  }
  // ---- tables shared by all grains: the quadrature and the m = 0 Wigner
  // set of every order of the loop, every m of every order a grain can end
  // at (cached in the context)
  std::vector<int> ngs;
  std::vector<std::pair<int, int>> keys;
  for (int k = kmin; k <= K; ++k) {
    ngs.push_back(glf * k);
    keys.push_back({k, glf * k});
  }
  std::vector<int> m0_sets, full_sets;
  if ((rc = ensure_gl(ctx, ngs)) || (rc = ensure_wigner(ctx, keys, false, m0_sets)) ||
      (rc = ensure_wigner(ctx, keys, true, full_sets))) {
    return rc;
  }
  // ---- item templates of every order: (m << 8 | class, class size), the
  // T-matrix size and the LU storage of a grain at that order, and the most
  // items of one grain in each size bucket
  std::vector<int32_t> tpl, tpl_off(K + 2, 0);
  std::vector<int64_t> tsz(K + 1, 0), lun(K + 1, 0);
  int64_t bmax[TMX_GM_BUCKETS] = {0, 0, 0, 0, 0};
  int nbmax_b[TMX_GM_BUCKETS] = {0, 0, 0, 0, 0};
  for (int N = 0; N <= K; ++N) {
    tpl_off[N] = (int32_t)(tpl.size() / 2);
    if (N < kmin) {
      continue;
    }
    int64_t bc[TMX_GM_BUCKETS] = {0, 0, 0, 0, 0};
    for (int m = 0; m <= N; ++m) {
      for (int cl = 0; cl < ((m == 0) ? 4 : 2); ++cl) {
        const int nb = tmx_host_class_size(N, m, cl);
        if (nb > 0) {
          tpl.push_back((m << 8) | cl);
          tpl.push_back(nb);
          const int b = gm_bucket(nb);
          bc[b] += 1;
          nbmax_b[b] = std::max(nbmax_b[b], nb);
          lun[N] += 2 * (int64_t)nb * nb;
        }
      }
    }
    for (int b = 0; b < TMX_GM_BUCKETS; ++b) {
      bmax[b] = std::max(bmax[b], bc[b]);
    }
    tsz[N] = tmx_tmatrix_size(N);
  }
  tpl_off[K + 1] = (int32_t)(tpl.size() / 2);
  // T-matrix and LU storage: the last batch's use (in either mode) with a
  // margin, else every grain at order 40 (at most every grain at the
  // largest order)
  const int kest = std::min(K, std::max(kmin, 40));
  const int64_t t_last = std::max(ctx->gm_last_t, ctx->p2_t_total);
  int64_t t_cap = std::max(ctx->gm_t_hint, t_last + t_last / 4);
  if (t_cap <= 0) {
    t_cap = n * tsz[kest];
  }
  // (at least what the T buffer already holds: the buffers only grow, and a
  // stable capacity keeps the graph's key, and so the graph, from changing
  // with every batch's T-matrix total)
  t_cap = std::max<int64_t>(t_cap, (int64_t)(ctx->T.cap / sizeof(cplx)));
  t_cap = std::min(t_cap, n * tsz[K]);
  int64_t lu_cap = std::max(ctx->gm_lu_hint, (int64_t)((double)t_cap * lun[K] / tsz[K]) + 2 * n * K * K);
  lu_cap = std::max<int64_t>(lu_cap, (int64_t)(ctx->gm_lu.cap / sizeof(cplx)));
  lu_cap = std::min(lu_cap, n * lun[K]);
  int32_t bcap[TMX_GM_BUCKETS];
  int64_t btot = 0;
  for (int b = 0; b < TMX_GM_BUCKETS; ++b) {
    bcap[b] = (int32_t)std::min<int64_t>(n * bmax[b], (int64_t)1 << 30);
    btot += bcap[b];
  }
  const int cmK = (Kg + 1) / 2;
  const int64_t arena_cap = (int64_t)(tab_per * n);
  const int nsteps = Kg - kmin + 1;
  // order-step slots: one per active grain, or a group's G orders of at most
  // 32 (G = 8) or 128 (G = 4) grains
  const int64_t ncap = std::max<int64_t>(
      n, std::max<int64_t>(8 * std::min<int64_t>(n, 32), 4 * std::min<int64_t>(n, 128)));
  // rounds: at least round_min grains final while the loop runs (at most
  // round_max of them), as in the host-driven loop
  const int round_min = (int)std::max<int64_t>(256, ctx->up_nact / 16);
  const int round_max = std::max(768, round_min);
  if ((rc = ensure(ctx, ctx->gm_state, sizeof(TmxGState))) ||
      (rc = ensure(ctx, ctx->gm_iter, sizeof(TmxGIter))) ||
      (rc = ensure(ctx, ctx->gm_steps, 2 * (size_t)nsteps * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->act0, n * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->act1, n * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->done, 2 * n * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->done_pos, n * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->keep_tab, n * sizeof(int64_t))) ||
      (rc = ensure(ctx, ctx->keep_q, n * sizeof(int64_t))) ||
      (rc = ensure(ctx, ctx->keep_ctl, 32)) ||
      (rc = ensure(ctx, ctx->keep_arena, arena_cap * sizeof(double))) ||
      (rc = ensure(ctx, ctx->gm_tab, ncap * (int64_t)glf * Kg * Kg * TMX_NQ * sizeof(double))) ||
      (rc = ensure(ctx, ctx->gm_nsc, ncap * (int64_t)glf * Kg * TMX_NS * sizeof(double))) ||
      (rc = ensure(ctx, ctx->gm_scr, 4 * ncap * 2 * (int64_t)cmK * cmK * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->gm_diag, ncap * 2 * (int64_t)Kg * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->gm_slots, ncap * sizeof(TmxSlot))) ||
      (rc = ensure(ctx, ctx->gm_items, 4 * ncap * sizeof(TmxItem))) ||
      (rc = ensure(ctx, ctx->gm_rslots, n * sizeof(TmxSlot))) ||
      (rc = ensure(ctx, ctx->gm_bitems, btot * sizeof(TmxItem))) ||
      (rc = ensure(ctx, ctx->gm_allitems, btot * sizeof(TmxItem))) ||
      (rc = ensure(ctx, ctx->gm_bptr, TMX_GM_BUCKETS * sizeof(TmxItem *))) ||
      (rc = ensure(ctx, ctx->gm_bcap, TMX_GM_BUCKETS * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->gm_tpl, std::max<size_t>(1, tpl.size()) * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->gm_tpl_off, tpl_off.size() * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->gm_full, full_sets.size() * sizeof(int32_t))) ||
      (rc = ensure(ctx, ctx->gm_tsize, tsz.size() * sizeof(int64_t))) ||
      (rc = ensure(ctx, ctx->gm_toff, n * sizeof(int64_t))) ||
      (rc = ensure(ctx, ctx->T, t_cap * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->gm_lu, lu_cap * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->gm_luscr, lu_cap * sizeof(cplx))) ||
      (rc = ensure(ctx, ctx->q, 2 * n * sizeof(double)))) {
    return rc;
  }
  TmxItem *bitems[TMX_GM_BUCKETS];
  {
    int64_t off = 0;
    for (int b = 0; b < TMX_GM_BUCKETS; ++b) {
      bitems[b] = (TmxItem *)ctx->gm_bitems.p + off;
      off += bcap[b];
    }
  }
  TmxGState *G = (TmxGState *)ctx->gm_state.p;
  TmxGIter *I = (TmxGIter *)ctx->gm_iter.p;
  int32_t *snap = (int32_t *)ctx->gm_steps.p;
  int32_t *outz = snap + nsteps;
  // ---- the graph, built again when the batch's shape or a buffer changed
  std::vector<uint64_t> key = {
      (uint64_t)n, (uint64_t)glf, (uint64_t)kmin, (uint64_t)K,
      (uint64_t)S.bessel_start, (uint64_t)t_cap, (uint64_t)lu_cap, (uint64_t)arena_cap,
      (uint64_t)round_min, (uint64_t)round_max, (uint64_t)Kg};
  uint64_t tol_bits;
  memcpy(&tol_bits, &S.tolerance, sizeof(tol_bits));
  key.push_back(tol_bits);
  for (int b = 0; b < TMX_GM_BUCKETS; ++b) {
    key.push_back((uint64_t)ctx->dispatch[b]);
    key.push_back((uint64_t)bcap[b]);
  }
  for (const DevBuf *b : {&ctx->gm_state, &ctx->gm_iter, &ctx->gm_steps, &ctx->act0,
                          &ctx->act1, &ctx->done, &ctx->done_pos, &ctx->keep_tab,
                          &ctx->keep_q, &ctx->keep_ctl, &ctx->keep_arena, &ctx->gm_tab,
                          &ctx->gm_nsc, &ctx->gm_scr, &ctx->gm_diag, &ctx->gm_slots,
                          &ctx->gm_items, &ctx->gm_rslots, &ctx->gm_bitems, &ctx->gm_bptr,
                          &ctx->gm_bcap, &ctx->gm_tpl, &ctx->gm_tpl_off, &ctx->gm_full,
                          &ctx->gm_tsize, &ctx->gm_toff, &ctx->T, &ctx->gm_lu,
                          &ctx->gm_luscr, &ctx->q, &ctx->state, &ctx->status, &ctx->grains,
                          &ctx->gl_x, &ctx->gl_w, &ctx->gl_off, &ctx->wig, &ctx->wig_off}) {
    key.push_back((uint64_t)(uintptr_t)b->p);
  }
  int nbk = 0; // size buckets a round launches
  for (int b = 0; b < TMX_GM_BUCKETS; ++b) {
    nbk += (bcap[b] > 0) ? 1 : 0;
  }
  if (key != ctx->gm_key || !ctx->gm_exec) {
    if (ctx->gm_exec) {
      CK(cudaGraphExecDestroy(ctx->gm_exec));
      ctx->gm_exec = nullptr;
    }
    if (ctx->gm_graph) {
      CK(cudaGraphDestroy(ctx->gm_graph));
      ctx->gm_graph = nullptr;
    }
    // the per-order tables the graph reads
    CK(cudaMemcpyAsync(ctx->gm_tpl.p, tpl.data(), tpl.size() * sizeof(int32_t),
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->gm_tpl_off.p, tpl_off.data(), tpl_off.size() * sizeof(int32_t),
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->gm_full.p, full_sets.data(), full_sets.size() * sizeof(int32_t),
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->gm_tsize.p, tsz.data(), tsz.size() * sizeof(int64_t),
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->gm_bptr.p, bitems, sizeof(bitems), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->gm_bcap.p, bcap, sizeof(bcap), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    int prio_lo = 0, prio_hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    if (!ctx->gm_cs) {
      // the loop chain's bodies are captured from a high-priority stream and
      // the rounds' from low-priority ones: captured kernels keep their
      // stream's priority, and the graph runs with per-node priorities
      CK(cudaStreamCreateWithPriority(&ctx->gm_cs, cudaStreamNonBlocking, prio_hi));
      CK(cudaStreamCreateWithPriority(&ctx->gm_rs, cudaStreamNonBlocking, prio_lo));
      for (cudaStream_t &x : ctx->gm_bs) {
        CK(cudaStreamCreateWithPriority(&x, cudaStreamNonBlocking, prio_lo));
      }
    }
    cudaGraph_t graph;
    CK(cudaGraphCreate(&graph, 0));
    ctx->gm_graph = graph;
    cudaStream_t cs = ctx->gm_cs, rs = ctx->gm_rs;
    std::vector<cudaEvent_t> evs;
    struct EvList {
      std::vector<cudaEvent_t> *v;
      ~EvList() {
        for (cudaEvent_t e : *v) {
          cudaEventDestroy(e);
        }
      }
    } ev_list{&evs};
    auto link = [&](cudaStream_t from, cudaStream_t to) -> int {
      cudaEvent_t e;
      CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      evs.push_back(e);
      CK(cudaEventRecord(e, from));
      CK(cudaStreamWaitEvent(to, e, 0));
      return 0;
    };
    // an IF node on `deps` whose body is captured from stream `s` by `body`
    auto add_if = [&](cudaGraphConditionalHandle h, cudaGraphNode_t dep, cudaStream_t s,
                      cudaGraphNode_t *node, const std::function<int()> &body) -> int {
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeIf;
      cp.conditional.size = 1;
      CK(cudaGraphAddNode(node, graph, &dep, 1, &cp));
      CK(cudaStreamBeginCaptureToGraph(s, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                       cudaStreamCaptureModeRelaxed));
      const int brc = body();
      cudaGraph_t captured = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(s, &captured);
      if (brc) {
        return brc;
      }
      CK(ce);
      return 0;
    };
    std::vector<cudaGraphNode_t> prev_loop;
    cudaGraphNode_t prev_form = nullptr, slot_exec[TMX_GM_RSLOTS] = {};
    for (int k = kmin; k <= Kg; ++k) {
      const int j = k - kmin;
      const int in = (j & 1) ? 2 : 0;
      const int out = 2 - in;
      int32_t *act_in = (int32_t *)((j & 1) ? ctx->act1.p : ctx->act0.p);
      int32_t *act_out = (int32_t *)((j & 1) ? ctx->act0.p : ctx->act1.p);
      // ---- loop chain: order step k, in one of three forms: this order
      // alone, or (few grains left) the group of orders k .. k + 3 or
      // k .. k + 7 where it fits below the last order
      const bool has4 = k + 3 <= Kg, has8 = k + 7 <= Kg;
      cudaGraphConditionalHandle hl, h4 = 0, h8 = 0;
      CK(cudaGraphConditionalHandleCreate(&hl, graph, 0, cudaGraphCondAssignDefault));
      if (has4) {
        CK(cudaGraphConditionalHandleCreate(&h4, graph, 0, cudaGraphCondAssignDefault));
      }
      if (has8) {
        CK(cudaGraphConditionalHandleCreate(&h8, graph, 0, cudaGraphCondAssignDefault));
      }
      cudaGraphNode_t e_node, l_node;
      if (tmx_gm_add_cond(graph, prev_loop.empty() ? nullptr : prev_loop.data(),
                          prev_loop.size(), &e_node, G, in, k, hl, h4, h8, has4 ? 1 : 0,
                          has8 ? 1 : 0, prio_hi)) {
        return fail(ctx, TMX_ERR_CUDA, "graph: step condition node");
      }
      auto step_body = [&]() -> int {
        tmx_launch_gm_begin(G, I, k, glf, m0_sets[j], in, out, cs);
        tmx_launch_gm_prep(&G->cnt[in], I, act_in, (int)n, (TmxSlot *)ctx->gm_slots.p,
                           (TmxItem *)ctx->gm_items.p, cs);
        tmx_launch_tables_dev((const TmxSlot *)ctx->gm_slots.p, (int)n, &G->cnt[in],
                              &I->ngauss, (const TmxGrain *)ctx->grains.p,
                              (const double *)ctx->gl_x.p, (const double *)ctx->gl_w.p,
                              (const int64_t *)ctx->gl_off.p, (double *)ctx->gm_tab.p,
                              (double *)ctx->gm_nsc.p, S.bessel_start, K, cs);
        TmxBlockArgs B;
        B.items = (const TmxItem *)ctx->gm_items.p;
        B.nitems = (int)(4 * n);
        B.range = I->m0_range;
        B.slots = (const TmxSlot *)ctx->gm_slots.p;
        B.grains = (const TmxGrain *)ctx->grains.p;
        B.tab = (const double *)ctx->gm_tab.p;
        B.nsc = (const double *)ctx->gm_nsc.p;
        B.wig = (const double *)ctx->wig.p;
        B.wig_off = (const int64_t *)ctx->wig_off.p;
        B.scratch = (cplx *)ctx->gm_scr.p;
        B.tout = nullptr;
        B.diag = (cplx *)ctx->gm_diag.p;
        B.status = (int32_t *)ctx->status.p;
        B.max_nb = (k + 1) / 2;
        B.chunk_nodes = tmx_host_chunk_nodes(B.max_nb);
        B.family = ctx->dispatch[gm_bucket(B.max_nb)];
        B.max_ctas = 148 * 8;
        tmx_launch_blocks(B, cs);
        tmx_launch_converge(act_in, (int)n, (const TmxSlot *)ctx->gm_slots.p,
                            (const cplx *)ctx->gm_diag.p, (TmxChainState *)ctx->state.p,
                            S.tolerance, k, K, act_out, &G->cnt[out], (int32_t *)ctx->done.p,
                            (int32_t *)ctx->done.p + n, (int32_t *)ctx->done_pos.p,
                            &G->cnt[1], &G->cnt[in], 0, cs);
        TmxKeepArgs KA;
        KA.done_list = (const int32_t *)ctx->done.p;
        KA.done_ord = (const int32_t *)ctx->done.p + n;
        KA.done_pos = (const int32_t *)ctx->done_pos.p;
        KA.counters = G->cnt;
        KA.next = (int32_t *)ctx->keep_ctl.p;
        KA.ticket = (unsigned *)ctx->keep_ctl.p + 1;
        KA.used = (unsigned long long *)ctx->keep_ctl.p + 1;
        KA.order0 = k;
        TmxChainBase &kb = KA.base[0];
        kb = TmxChainBase{};
        kb.tab_stride = (int64_t)glf * k * k * TMX_NQ;
        kb.nsc_stride = (int64_t)glf * k * TMX_NS;
        kb.diag_stride = 2 * (int64_t)k;
        kb.scr_stride = 2 * (int64_t)((k + 1) / 2) * ((k + 1) / 2);
        KA.tab = (const double *)ctx->gm_tab.p;
        KA.nsc = (const double *)ctx->gm_nsc.p;
        KA.arena = (double *)ctx->keep_arena.p;
        KA.cap = arena_cap;
        KA.keep_tab = (int64_t *)ctx->keep_tab.p;
        KA.keep_q = (int64_t *)ctx->keep_q.p;
        tmx_launch_keep_tables(KA, (int)n, cs);
        tmx_launch_gm_step_end(G, snap, outz, j, out, -1, k + 1, 7, cs);
        CK(cudaGetLastError());
        return 0;
      };
      if ((rc = add_if(hl, e_node, cs, &l_node, step_body))) {
        return rc;
      }
      prev_loop.assign(1, l_node);
      // the group of orders k .. k + gk - 1 for at most `chunk` active
      // grains, laid out as the host-driven loop's speculative groups: slots
      // [s chunk, (s + 1) chunk) for order k + s, positions past the list's
      // length empty; after the group its surviving list becomes the input
      // list of order k + gk (the same parity)
      auto group_body = [&](int gk, int chunk) -> int {
        TmxChainBase base[TMX_MAX_GROUP];
        int64_t tab_t = 0, nsc_t = 0, diag_t = 0, scr_t = 0;
        for (int q = 0; q < gk; ++q) {
          const int ks = k + q;
          const int cm = (ks + 1) / 2;
          TmxChainBase &b = base[q];
          b.tab_stride = (int64_t)glf * ks * ks * TMX_NQ;
          b.nsc_stride = (int64_t)glf * ks * TMX_NS;
          b.diag_stride = 2 * (int64_t)ks;
          b.scr_stride = 2 * (int64_t)cm * cm;
          b.slot = q * chunk;
          b.tab = tab_t;
          b.nsc = nsc_t;
          b.diag = diag_t;
          b.scr = scr_t;
          tab_t += chunk * b.tab_stride;
          nsc_t += chunk * b.nsc_stride;
          diag_t += chunk * b.diag_stride;
          scr_t += 4 * chunk * b.scr_stride;
        }
        for (int q = 0; q < gk; ++q) {
          tmx_launch_chain_prep(act_in, chunk, &G->cnt[in], 0, k + q, glf * (k + q),
                                m0_sets[j + q], base[q], (TmxSlot *)ctx->gm_slots.p,
                                (TmxItem *)ctx->gm_items.p, cs);
        }
        const int kl = k + gk - 1;
        tmx_launch_tables((const TmxSlot *)ctx->gm_slots.p, gk * chunk,
                          (const TmxGrain *)ctx->grains.p, (const double *)ctx->gl_x.p,
                          (const double *)ctx->gl_w.p, (const int64_t *)ctx->gl_off.p,
                          (double *)ctx->gm_tab.p, (double *)ctx->gm_nsc.p, S.bessel_start,
                          glf * kl, kl, cs);
        TmxBlockArgs B;
        B.items = (const TmxItem *)ctx->gm_items.p;
        B.nitems = 4 * gk * chunk;
        B.slots = (const TmxSlot *)ctx->gm_slots.p;
        B.grains = (const TmxGrain *)ctx->grains.p;
        B.tab = (const double *)ctx->gm_tab.p;
        B.nsc = (const double *)ctx->gm_nsc.p;
        B.wig = (const double *)ctx->wig.p;
        B.wig_off = (const int64_t *)ctx->wig_off.p;
        B.scratch = (cplx *)ctx->gm_scr.p;
        B.tout = nullptr;
        B.diag = (cplx *)ctx->gm_diag.p;
        B.status = (int32_t *)ctx->status.p;
        B.max_nb = (kl + 1) / 2;
        B.chunk_nodes = tmx_host_chunk_nodes(B.max_nb);
        B.family = ctx->dispatch[gm_bucket(B.max_nb)];
        tmx_launch_blocks(B, cs);
        for (int q = 0; q < gk; ++q) {
          // (the output list after the group is the one of its last order)
          CK(cudaMemsetAsync(&G->cnt[out], 0, sizeof(int32_t), cs));
          tmx_launch_converge(act_in, chunk, (const TmxSlot *)ctx->gm_slots.p + base[q].slot,
                              (const cplx *)ctx->gm_diag.p, (TmxChainState *)ctx->state.p,
                              S.tolerance, k + q, K, act_out, &G->cnt[out],
                              (int32_t *)ctx->done.p, (int32_t *)ctx->done.p + n,
                              (int32_t *)ctx->done_pos.p, &G->cnt[1], &G->cnt[in], 0, cs);
        }
        TmxKeepArgs KA;
        KA.done_list = (const int32_t *)ctx->done.p;
        KA.done_ord = (const int32_t *)ctx->done.p + n;
        KA.done_pos = (const int32_t *)ctx->done_pos.p;
        KA.counters = G->cnt;
        KA.next = (int32_t *)ctx->keep_ctl.p;
        KA.ticket = (unsigned *)ctx->keep_ctl.p + 1;
        KA.used = (unsigned long long *)ctx->keep_ctl.p + 1;
        KA.order0 = k;
        for (int q = 0; q < gk; ++q) {
          KA.base[q] = base[q];
        }
        KA.tab = (const double *)ctx->gm_tab.p;
        KA.nsc = (const double *)ctx->gm_nsc.p;
        KA.arena = (double *)ctx->keep_arena.p;
        KA.cap = arena_cap;
        KA.keep_tab = (int64_t *)ctx->keep_tab.p;
        KA.keep_q = (int64_t *)ctx->keep_q.p;
        tmx_launch_keep_tables(KA, (int)n, cs);
        tmx_launch_gm_relist(G, act_out, act_in, (int)n, in, out, cs);
        tmx_launch_gm_step_end(G, snap, outz, j, out, in, k + gk, 2 * gk + 5, cs);
        CK(cudaGetLastError());
        return 0;
      };
      for (int f = 0; f < 2; ++f) {
        const int gk = f ? 8 : 4;
        if (!(f ? has8 : has4)) {
          continue;
        }
        cudaGraphNode_t g_node;
        if ((rc = add_if(f ? h8 : h4, e_node, cs, &g_node,
                         [&]() { return group_body(gk, (int)std::min<int64_t>(n, f ? 32 : 128)); }))) {
          return rc;
        }
        prev_loop.push_back(g_node);
      }
      // ---- round chain: the blocks of the grains final so far. Rounds are
      // formed one after another (item lists, T-matrix and LU offsets from
      // shared counters) and run in round slots k mod TMX_GM_RSLOTS, so that
      // a round's blocks overlap the next rounds' (the host-driven loop's
      // rounds overlap on two streams); a slot is reused only after its
      // previous round, TMX_GM_RSLOTS orders earlier, is done
      const int rsl = j % TMX_GM_RSLOTS;
      cudaGraphConditionalHandle hform, hexec;
      CK(cudaGraphConditionalHandleCreate(&hform, graph, 0, cudaGraphCondAssignDefault));
      CK(cudaGraphConditionalHandleCreate(&hexec, graph, 0, cudaGraphCondAssignDefault));
      cudaGraphNode_t f_node, form_node, exec_node;
      std::vector<cudaGraphNode_t> fdeps = prev_loop;
      if (prev_form) {
        fdeps.push_back(prev_form);
      }
      if (slot_exec[rsl]) {
        // (the slot's previous round must be done before its state is reused)
        fdeps.push_back(slot_exec[rsl]);
      }
      if (tmx_gm_add_decide(graph, fdeps.data(), fdeps.size(), &f_node, G, snap, outz, j,
                            k == Kg ? 1 : 0, round_min, round_max, rsl, hform, hexec,
                            prio_hi)) {
        return fail(ctx, TMX_ERR_CUDA, "graph: round condition node");
      }
      auto form_body = [&]() -> int {
        TmxGmRoundArgs RA;
        RA.G = G;
        RA.rs = rsl;
        RA.done_list = (const int32_t *)ctx->done.p;
        RA.done_ord = (const int32_t *)ctx->done.p + n;
        RA.keep_tab = (const int64_t *)ctx->keep_tab.p;
        RA.tpl_off = (const int32_t *)ctx->gm_tpl_off.p;
        RA.tpl = (const int32_t *)ctx->gm_tpl.p;
        RA.full_sets = (const int32_t *)ctx->gm_full.p;
        RA.tsize = (const int64_t *)ctx->gm_tsize.p;
        RA.glf = glf;
        RA.min_order = kmin;
        RA.rslots = (TmxSlot *)ctx->gm_rslots.p;
        RA.n = (int)n;
        RA.bitems = (TmxItem *const *)ctx->gm_bptr.p;
        RA.bcap = (const int32_t *)ctx->gm_bcap.p;
        RA.t_off = (int64_t *)ctx->gm_toff.p;
        RA.t_cap = (unsigned long long)t_cap;
        RA.lu_cap = (unsigned long long)lu_cap;
        tmx_launch_gm_round(RA, cs);
        tmx_launch_gm_round_mid(G, rsl, cs);
        tmx_launch_gm_tzero(G, rsl, (const TmxSlot *)ctx->gm_rslots.p,
                            (const int64_t *)ctx->gm_tsize.p, (cplx *)ctx->T.p, cs);
        CK(cudaGetLastError());
        return 0;
      };
      // (the formation is short: its kernels run at the loop's priority, so
      // that they do not queue behind the running round's blocks)
      if ((rc = add_if(hform, f_node, cs, &form_node, form_body))) {
        return rc;
      }
      auto exec_body = [&]() -> int {
        for (int b = TMX_GM_BUCKETS - 1; b >= 0; --b) {
          if (bcap[b] == 0) {
            continue;
          }
          cudaStream_t bs = ctx->gm_bs[b];
          int lrc;
          if ((lrc = link(rs, bs))) {
            return lrc;
          }
          TmxBlockArgs R;
          R.items = bitems[b];
          R.nitems = bcap[b];
          R.range = &G->rng[rsl][b][0];
          R.slots = (const TmxSlot *)ctx->gm_rslots.p;
          R.grains = (const TmxGrain *)ctx->grains.p;
          R.tab = (const double *)ctx->keep_arena.p;
          R.nsc = (const double *)ctx->keep_arena.p;
          R.wig = (const double *)ctx->wig.p;
          R.wig_off = (const int64_t *)ctx->wig_off.p;
          R.scratch = (cplx *)ctx->gm_luscr.p;
          R.tout = (cplx *)ctx->T.p;
          R.diag = nullptr;
          R.status = (int32_t *)ctx->status.p;
          R.max_nb = nbmax_b[b];
          R.chunk_nodes = tmx_host_chunk_nodes(R.max_nb);
          R.lu = (cplx *)ctx->gm_lu.p;
          R.family = ctx->dispatch[b];
          R.max_ctas = TMX_GM_ROUND_CTAS;
          tmx_launch_blocks(R, bs);
        }
        // (joined only after every bucket has forked, so that they run
        // side by side)
        for (int b = 0; b < TMX_GM_BUCKETS; ++b) {
          int lrc;
          if (bcap[b] > 0 && (lrc = link(ctx->gm_bs[b], rs))) {
            return lrc;
          }
        }
        tmx_launch_qsums((const TmxSlot *)ctx->gm_rslots.p, (int)n, (const cplx *)ctx->T.p,
                         (double *)ctx->q.p, rs, &G->srng[rsl][0], 148 * 4);
        tmx_launch_gm_round_end(G, 5 + nbk, rs);
        CK(cudaGetLastError());
        return 0;
      };
      if ((rc = add_if(hexec, form_node, rs, &exec_node, exec_body))) {
        return rc;
      }
      prev_form = form_node;
      slot_exec[rsl] = exec_node;
    }
    CK(cudaGraphInstantiateWithFlags(&ctx->gm_exec, graph,
                                     cudaGraphInstantiateFlagUseNodePriority));
    ctx->gm_key = key;
  }
  // ---- this batch: initial state, the graph, the results
  TmxGState g0 = {};
  g0.cnt[0] = ctx->up_nact;
  g0.next_k = kmin;
  CK(cudaMemcpyAsync(G, &g0, sizeof(g0), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(snap, 0xff, nsteps * sizeof(int32_t), st));
  CK(cudaMemsetAsync(outz, 0, nsteps * sizeof(int32_t), st));
  CK(cudaMemcpyAsync(ctx->state.p, ctx->state0.p, n * sizeof(TmxChainState),
                     cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(ctx->act0.p, ctx->actinit.p, ctx->up_nact * sizeof(int32_t),
                     cudaMemcpyDeviceToDevice, st));
  CK(cudaMemsetAsync(ctx->status.p, 0, n * sizeof(int32_t), st));
  CK(cudaMemsetAsync(ctx->keep_ctl.p, 0, 32, st));
  CK(cudaMemsetAsync(ctx->gm_toff.p, 0xff, n * sizeof(int64_t), st));
  CK(cudaGraphLaunch(ctx->gm_exec, st));
  CK(cudaGetLastError());
  // the per-grain results and the round items (for the gradients) follow
  // the graph on the same stream: one synchronisation
  TmxGState g1;
  std::vector<TmxChainState> st0(n);
  std::vector<int64_t> toff(n);
  std::vector<double> q2(2 * n);
  std::vector<int32_t> stb(n);
  CK(cudaMemcpyAsync(&g1, G, sizeof(g1), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(st0.data(), ctx->state.p, n * sizeof(TmxChainState),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(toff.data(), ctx->gm_toff.p, n * sizeof(int64_t),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(q2.data(), ctx->q.p, 2 * n * sizeof(double), cudaMemcpyDeviceToHost,
                     st));
  CK(cudaMemcpyAsync(stb.data(), ctx->status.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                     st));
  {
    // every bucket's item array at its capacity, largest bucket first (the
    // fill counts are known only after the graph)
    int64_t off = 0;
    for (int b = TMX_GM_BUCKETS - 1; b >= 0; --b) {
      if (bcap[b] > 0) {
        CK(cudaMemcpyAsync((TmxItem *)ctx->gm_allitems.p + off, bitems[b],
                           bcap[b] * sizeof(TmxItem), cudaMemcpyDeviceToDevice, st));
      }
      off += bcap[b];
    }
  }
  CK(cudaStreamSynchronize(st));
  // kernels the graph ran: the two control nodes of every order, the
  // bodies of the steps and rounds that ran
  ctx->launches += 2 * (int64_t)nsteps + (int64_t)g1.kernels;
  if (g1.overflow || g1.cnt[1] != ctx->up_nact || g1.cursor != g1.cnt[1]) {
    // storage ran out (or a grain was not finished): grow the estimates and
    // compute this batch in the host mode
    ctx->gm_t_hint = std::max<int64_t>(2 * t_cap, (int64_t)g1.t_used + (int64_t)g1.t_used / 4);
    ctx->gm_lu_hint = std::max<int64_t>(2 * lu_cap, (int64_t)g1.lu_used + (int64_t)g1.lu_used / 4);
    return 1;
  }
  ctx->gm_counts[0] = g1.steps;
  ctx->gm_counts[1] = g1.rounds;
  for (int64_t i = 0; i < n; ++i) {
    ctx->nmax_h[i] = st0[i].nmax;
    ctx->ngauss_h[i] = st0[i].ngauss;
    ctx->status_h[i] = st0[i].status | ctx->up_status[i];
    ctx->q_h[6 * i + 0] = st0[i].qsca;
    ctx->q_h[6 * i + 1] = st0[i].qext;
    ctx->q_h[6 * i + 4] = st0[i].dqs;
    ctx->q_h[6 * i + 5] = st0[i].dqe;
    ctx->t_off_h[i] = (st0[i].nmax > 0) ? toff[i] : 0;
  }
  // the rounds' items in one array, largest size bucket first, with their
  // class sizes, for the gradients (their LU factors stay in gm_lu)
  tmx_ctx::RoundRec rec;
  rec.own_tables = false;
  rec.borrowed = true;
  rec.tab = rec.nsc = (double *)ctx->keep_arena.p;
  rec.slots = (TmxSlot *)ctx->gm_rslots.p;
  rec.items = (TmxItem *)ctx->gm_allitems.p;
  rec.lu = (cplx *)ctx->gm_lu.p;
  rec.scr_total = (int64_t)g1.lu_used;
  {
    int64_t off = 0;
    for (int b = TMX_GM_BUCKETS - 1; b >= 0; --b) {
      const int64_t c = std::min(g1.fill[b], bcap[b]);
      if (c > 0) {
        rec.seg.push_back({off, off + c, (int64_t)nbmax_b[b]});
      }
      off += bcap[b];
    }
  }
  ctx->rounds_kept.push_back(std::move(rec));
  ctx->gm_last_t = (int64_t)g1.t_used;
  ctx->sink_done = 0;
  if ((rc = finish_blocks(ctx, (int64_t)g1.t_used, 1, &q2, &stb))) {
    return rc;
  }
  ctx->rounds_lu = true;
  ctx->last_mode = TMX_BATCH_GRAPH;
  return TMX_OK;
}

extern "C" int tmx_set_batch_mode(tmx_ctx *ctx, int mode) {
  if (!ctx || (mode != TMX_BATCH_HOST && mode != TMX_BATCH_GRAPH)) {
    return TMX_ERR_INVALID;
  }
  ctx->batch_mode = mode;
  return TMX_OK;
}

extern "C" int tmx_get_batch_mode(tmx_ctx *ctx, int *mode) {
  if (!ctx || !mode) {
    return TMX_ERR_INVALID;
  }
  *mode = ctx->batch_mode;
  return TMX_OK;
}

extern "C" int tmx_last_batch_mode(tmx_ctx *ctx, int *mode) {
  if (!ctx || !mode) {
    return TMX_ERR_INVALID;
  }
  *mode = ctx->last_mode;
  return TMX_OK;
}

static double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
      .count();
}

int tmx_batch_compute(tmx_ctx *ctx) {
  if (!ctx) {
    return TMX_ERR_INVALID;
  }
  if (!ctx->uploaded) {
    return fail(ctx, TMX_ERR_STATE, "no batch uploaded");
  }
  struct WallClock {
    tmx_ctx *c;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    ~WallClock() { c->host_times[0] = ms_since(t0); }
  } wall{ctx};
  ctx->host_times[1] = ctx->host_times[2] = ctx->host_times[3] = 0.;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int64_t n = ctx->up_n;
  const tmx_schedule S = ctx->up_sched;
  const int glf = S.gauss_legendre_factor;
  int rc;
  ctx->have_batch = false;
  ctx->lu_ready = false;
  if ((rc = tmx_release_rounds(ctx))) {
    return rc;
  }
  ctx->n = n;
  ++ctx->batch_seq;
  ctx->nmax_h.assign(n, 0);
  ctx->ngauss_h.assign(n, 0);
  ctx->status_h.assign(n, 0);
  ctx->q_h.assign(6 * n, 0.);
  ctx->t_off_h.assign(n, 0);
  ctx->flops_survey = 0.;
  if (n == 0) {
    ctx->p2_t_total = 0;
    ctx->have_batch = true;
    return TMX_OK;
  }
  ctx->last_mode = TMX_BATCH_HOST;
  if (ctx->batch_mode == TMX_BATCH_GRAPH) {
    rc = gm_compute(ctx);
    if (rc != 1) {
      if (rc == TMX_OK) {
        note_kmax(ctx);
      }
      return rc;
    }
  }
  std::vector<TmxChainState> st0(n);
  if ((rc = tl_mark(ctx, TMX_TL_BATCH_START, st))) {
    return rc;
  }
  CK(cudaMemcpyAsync(ctx->state.p, ctx->state0.p, n * sizeof(TmxChainState),
                     cudaMemcpyDeviceToDevice, st));
  if (ctx->up_nact > 0) {
    CK(cudaMemcpyAsync(ctx->act0.p, ctx->actinit.p,
                       ctx->up_nact * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                       st));
  }
  CK(cudaMemsetAsync(ctx->status.p, 0, n * sizeof(int32_t), st));

  // ---- tables shared by all grains
  std::vector<int> ngs;
  std::vector<std::pair<int, int>> chain_keys;
  for (int k = S.min_order; k < S.max_order; ++k) {
    ngs.push_back(glf * k);
    chain_keys.push_back({k, glf * k});
  }
  if ((rc = ensure_gl(ctx, ngs))) {
    return rc;
  }
  std::vector<int> chain_sets;
  if ((rc = ensure_wigner(ctx, chain_keys, false, chain_sets))) {
    return rc;
  }
  {
    // every m of the orders the blocks of most grains run at, made before
    // the loop (cached in the context), so that block rounds need not wait
    // for table jobs queued behind the order loop
    std::vector<std::pair<int, int>> full_keys;
    for (int k = S.min_order; k < std::min(S.max_order, 65); ++k) {
      full_keys.push_back({k, glf * k});
    }
    std::vector<int> full_sets;
    if ((rc = ensure_wigner(ctx, full_keys, true, full_sets))) {
      return rc;
    }
  }

  // ---- 1. order loop
  // Grains whose order became final are collected from the done list after
  // every order; once enough are ready, their blocks run as a round on the
  // second (lower-priority) stream while the order loop continues, so the
  // blocks fill the GPU during the latency-bound tail of the loop. A round's
  // host set-up is issued after the next order's launches, so it overlaps
  // that order on the GPU.
  // done list: grains [0, n) and their final orders [n, 2n)
  if ((rc = ensure(ctx, ctx->done, std::max<int64_t>(1, 2 * n) * sizeof(int32_t)))) {
    return rc;
  }
  if (ctx->pinned_done_cap < 2 * n) {
    if (ctx->pinned_done) {
      CK(cudaFreeHost(ctx->pinned_done));
      ctx->pinned_done = nullptr;
      ctx->pinned_done_cap = 0;
    }
    CK(cudaMallocHost((void **)&ctx->pinned_done, 2 * n * sizeof(int32_t)));
    ctx->pinned_done_cap = 2 * n;
  }
  CK(cudaMemsetAsync(ctx->count.p, 0, 2 * sizeof(int32_t), st));
  // arena for the final-order tables of every grain (k_keep_tables): sized
  // from the last batch's use, else for orders up to 40; at most 8 GiB. A
  // grain that does not fit keeps no copy and its round computes its tables.
  ctx->keep_valid = false;
  int64_t keep_cap = 0;
  {
    const int64_t topk = std::min(S.max_order - 1, 40);
    const int64_t per = glf * topk * topk * TMX_NQ + glf * topk * TMX_NS + 32;
    keep_cap = std::max<int64_t>(ctx->keep_used_last + ctx->keep_used_last / 4,
                                 std::min<int64_t>(n * per, (int64_t)1 << 27));
    keep_cap = std::min<int64_t>(keep_cap, (int64_t)1 << 30);
    if ((rc = ensure(ctx, ctx->keep_arena, keep_cap * sizeof(double))) ||
        (rc = ensure(ctx, ctx->keep_tab, n * sizeof(int64_t))) ||
        (rc = ensure(ctx, ctx->keep_q, n * sizeof(int64_t))) ||
        (rc = ensure(ctx, ctx->done_pos, n * sizeof(int32_t))) ||
        (rc = ensure(ctx, ctx->keep_ctl, 32))) {
      return rc;
    }
    CK(cudaMemsetAsync(ctx->keep_ctl.p, 0, 32, st));
    if (ctx->pinned_keep_cap < n) {
      if (ctx->pinned_keep) {
        CK(cudaFreeHost(ctx->pinned_keep));
        ctx->pinned_keep = nullptr;
        ctx->pinned_keep_cap = 0;
      }
      CK(cudaMallocHost((void **)&ctx->pinned_keep, n * sizeof(int64_t)));
      ctx->pinned_keep_cap = n;
    }
    ctx->keep_off_h.assign(n, -1);
    ctx->keep_valid = true;
  }
  // the rounds of this batch keep their buffers and LU factors
  struct KeepGuard {
    tmx_ctx *c;
    ~KeepGuard() { c->keep_rounds = false; }
  } keep_guard{ctx};
  ctx->keep_rounds = true;
  const int64_t round_min = std::max<int64_t>(256, ctx->up_nact / 16);
  const int64_t round_max = std::max<int64_t>(768, round_min);
  int64_t done_seen = 0;
  std::vector<int32_t> ready, pending;
  std::vector<char> launched(n, 0);
  int rounds = 0;
  int64_t t_next = 0;
  const size_t budget = (size_t)8 << 30; // table bytes per chunk
  std::unique_ptr<NvtxRange> chain_range(new NvtxRange("tmx_chain"));
  const int last = S.max_order - 1;
  // The loop runs one group of orders ahead of the host: group j + 1 is
  // queued before the host waits for group j's outcome, with the length of
  // its active list read on the device (the host launches for an upper
  // bound, the input length of group j; surplus positions are empty
  // slots). So the GPU never waits for the host between orders; the host
  // reads each group's counts and done-list entries while the next group
  // runs. Active lists alternate between act0 and act1; their lengths are
  // count[0] and count[2], the done-list length count[1].
  DevBuf *lists[2] = {&ctx->act0, &ctx->act1};
  int32_t *cnt = (int32_t *)ctx->count.p;
  ctx->pinned[12] = ctx->up_nact;
  CK(cudaMemcpyAsync(cnt, ctx->pinned + 12, sizeof(int32_t), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(cnt + 2, 0, sizeof(int32_t), st));
  struct Group {
    int k = 0, G = 0;
    int nact_up = 0; // upper bound of the group's input list length
    int issued = 0;  // the bound it was launched for
    int list = 0, par = 0;
  };
  cudaEvent_t gev[2];
  CK(cudaEventCreateWithFlags(&gev[0], cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&gev[1], cudaEventDisableTiming));
  struct EvGuard {
    cudaEvent_t *e;
    ~EvGuard() {
      cudaEventDestroy(e[0]);
      cudaEventDestroy(e[1]);
    }
  } ev_guard{gev};
  int64_t unprocessed_bound = 0; // done entries groups in flight may add
  auto issue = [&](Group &grp) -> int {
    const int k = grp.k, G = grp.G, nact = grp.nact_up;
    grp.issued = nact;
    const int32_t *cur_cnt = cnt + (grp.list ? 2 : 0);
    int32_t *nxt_cnt = cnt + (grp.list ? 0 : 2);
    DevBuf *cur = lists[grp.list], *nxt = lists[grp.list ^ 1];
    std::vector<TmxChainBase> base(G);
    int64_t tab_t = 0, nsc_t = 0, diag_t = 0, scr_t = 0;
    int chunk = nact;
    for (int s = 0; s < G; ++s) {
      const int ks = k + s;
      const int cm = (ks + 1) / 2;
      TmxChainBase &b = base[s];
      b.tab_stride = (int64_t)glf * ks * ks * TMX_NQ;
      b.nsc_stride = (int64_t)glf * ks * TMX_NS;
      b.diag_stride = 2 * (int64_t)ks;
      b.scr_stride = 2 * (int64_t)cm * cm;
      if (G == 1) {
        const size_t per_slot = (b.tab_stride + b.nsc_stride) * sizeof(double) +
                                (4 * b.scr_stride + b.diag_stride) * sizeof(cplx);
        chunk = (int)std::max<size_t>(1, std::min<size_t>(nact, budget / per_slot));
      }
      b.slot = s * chunk;
      b.tab = tab_t;
      b.nsc = nsc_t;
      b.diag = diag_t;
      b.scr = scr_t;
      tab_t += chunk * b.tab_stride;
      nsc_t += chunk * b.nsc_stride;
      diag_t += chunk * b.diag_stride;
      scr_t += 4 * chunk * b.scr_stride;
    }
    int rc2;
    if ((rc2 = ensure(ctx, ctx->tab, tab_t * sizeof(double))) ||
        (rc2 = ensure(ctx, ctx->nsc, nsc_t * sizeof(double))) ||
        (rc2 = ensure(ctx, ctx->scratch, scr_t * sizeof(cplx))) ||
        (rc2 = ensure(ctx, ctx->diag, diag_t * sizeof(cplx))) ||
        (rc2 = ensure(ctx, ctx->slots, (size_t)G * chunk * sizeof(TmxSlot))) ||
        (rc2 = ensure(ctx, ctx->items, 4 * (size_t)G * chunk * sizeof(TmxItem)))) {
      return rc2;
    }
    CK(cudaMemsetAsync(nxt_cnt, 0, sizeof(int32_t), st));
    const int kl = k + G - 1;
    for (int c0 = 0; c0 < nact; c0 += chunk) {
      const int cn = std::min(chunk, nact - c0);
      const int32_t *a = (const int32_t *)cur->p + c0;
      for (int s = 0; s < G; ++s) {
        tmx_launch_chain_prep(a, cn, cur_cnt, c0, k + s, glf * (k + s),
                              chain_sets[k + s - S.min_order], base[s],
                              (TmxSlot *)ctx->slots.p, (TmxItem *)ctx->items.p, st);
        LAUNCHED();
      }
      // slots and items of the group are contiguous: [s][p]
      const int nsl = (G == 1) ? cn : G * chunk;
      cudaEvent_t pe = nullptr;
      if ((rc2 = prof_begin(ctx, 1, &pe))) {
        return rc2;
      }
      tmx_launch_tables((const TmxSlot *)ctx->slots.p, nsl,
                        (const TmxGrain *)ctx->grains.p,
                        (const double *)ctx->gl_x.p, (const double *)ctx->gl_w.p,
                        (const int64_t *)ctx->gl_off.p, (double *)ctx->tab.p,
                        (double *)ctx->nsc.p, S.bessel_start, glf * kl, kl, st);
      LAUNCHED();
      if ((rc2 = prof_end(ctx, 1, pe, 0., nullptr, 0., nsl))) {
        return rc2;
      }
      TmxBlockArgs B;
      B.items = (const TmxItem *)ctx->items.p;
      B.nitems = 4 * nsl;
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
      B.max_nb = (kl + 1) / 2;
      B.chunk_nodes = tmx_host_chunk_nodes(B.max_nb);
      B.family = dispatch_family(ctx, B.max_nb);
      // (flops of the upper bound of slots: the profiled figure is an
      // estimate until the group's length is known)
      double fl = 0.;
      for (int s = 0; s < G; ++s) {
        for (int c = 0; c < 4; ++c) {
          fl += item_flops(tmx_host_class_size(k + s, 0, c), 0, glf * (k + s)) * cn;
        }
      }
      if ((rc2 = prof_begin(ctx, 0, &pe))) {
        return rc2;
      }
      tmx_launch_blocks(B, st);
      LAUNCHED();
      if ((rc2 = prof_end(ctx, 0, pe, fl, nullptr, 0., B.nitems))) {
        return rc2;
      }
      for (int s = 0; s < G; ++s) {
        if (G > 1) {
          // the active list after the group is the one of its last order
          CK(cudaMemsetAsync(nxt_cnt, 0, sizeof(int32_t), st));
        }
        tmx_launch_converge(a, cn, (const TmxSlot *)ctx->slots.p + base[s].slot,
                            (const cplx *)ctx->diag.p,
                            (TmxChainState *)ctx->state.p, S.tolerance, k + s, last,
                            (int32_t *)nxt->p, nxt_cnt, (int32_t *)ctx->done.p,
                            (int32_t *)ctx->done.p + n, (int32_t *)ctx->done_pos.p,
                            cnt + 1, cur_cnt, c0, st);
        LAUNCHED();
      }
      if (ctx->keep_valid) {
        // the tables of the grains this chunk made final, before the next
        // chunk or group overwrites them
        TmxKeepArgs K;
        K.done_list = (const int32_t *)ctx->done.p;
        K.done_ord = (const int32_t *)ctx->done.p + n;
        K.done_pos = (const int32_t *)ctx->done_pos.p;
        K.counters = cnt;
        K.next = (int32_t *)ctx->keep_ctl.p;
        K.ticket = (unsigned *)ctx->keep_ctl.p + 1;
        K.used = (unsigned long long *)ctx->keep_ctl.p + 1;
        K.order0 = k;
        for (int s = 0; s < G; ++s) {
          K.base[s] = base[s];
        }
        K.tab = (const double *)ctx->tab.p;
        K.nsc = (const double *)ctx->nsc.p;
        K.arena = (double *)ctx->keep_arena.p;
        K.cap = keep_cap;
        K.keep_tab = (int64_t *)ctx->keep_tab.p;
        K.keep_q = (int64_t *)ctx->keep_q.p;
        tmx_launch_keep_tables(K, cn, st);
        LAUNCHED();
      }
    }
    // the group's outcome for the host: the new list length and the
    // done-list length (pinned slots of this group's parity), and every
    // done-list entry that the groups in flight can have added
    unprocessed_bound += nact;
    const int64_t w = std::min<int64_t>(n - done_seen, unprocessed_bound);
    CK(cudaMemcpyAsync(ctx->pinned + 8 + 2 * grp.par, nxt_cnt, sizeof(int32_t),
                       cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(ctx->pinned + 9 + 2 * grp.par, cnt + 1, sizeof(int32_t),
                       cudaMemcpyDeviceToHost, st));
    if (w > 0) {
      CK(cudaMemcpyAsync(ctx->pinned_done + done_seen, (int32_t *)ctx->done.p + done_seen,
                         w * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(ctx->pinned_done + n + done_seen,
                         (int32_t *)ctx->done.p + n + done_seen, w * sizeof(int32_t),
                         cudaMemcpyDeviceToHost, st));
      if (ctx->keep_valid) {
        CK(cudaMemcpyAsync(ctx->pinned_keep + done_seen,
                           (int64_t *)ctx->keep_q.p + done_seen, w * sizeof(int64_t),
                           cudaMemcpyDeviceToHost, st));
      }
    }
    CK(cudaEventRecord(gev[grp.par], st));
    return TMX_OK;
  };
  // speculative group length for a list of at most nact grains: few grains
  // left -- evaluate the next G orders of every active grain at once (the
  // convergence rule is then applied order by order), which cuts the
  // latency-bound tail at the cost of orders past convergence
  auto group_len = [&](int k, int nact) {
    return std::min(S.max_order - k, nact <= 32 ? 8 : (nact <= 128 ? 4 : 1));
  };
  Group inflight;
  bool have_inflight = false;
  if (ctx->up_nact > 0) {
    inflight.k = S.min_order;
    inflight.nact_up = ctx->up_nact;
    inflight.G = group_len(inflight.k, inflight.nact_up);
    inflight.list = 0;
    inflight.par = 0;
    if ((rc = issue(inflight))) {
      return rc;
    }
    have_inflight = true;
  }
  int nact_known = ctx->up_nact;
  while (have_inflight) {
    // queue the next group before waiting for this one
    Group next;
    bool have_next = false;
    const int k_next = inflight.k + inflight.G;
    if (k_next < S.max_order && nact_known > 0) {
      next.k = k_next;
      next.nact_up = inflight.nact_up; // the list can only shrink
      next.G = group_len(next.k, next.nact_up);
      next.list = inflight.list ^ 1;
      next.par = inflight.par ^ 1;
      if ((rc = issue(next))) {
        return rc;
      }
      have_next = true;
    }
    // a round's host set-up overlaps the groups on the GPU
    if (!pending.empty()) {
      const auto tr = std::chrono::steady_clock::now();
      if ((rc = run_blocks_round(ctx, pending, (rounds & 1) ? ctx->stream3 : ctx->stream2,
                                 t_next, rounds > 0, &t_next, true))) {
        return rc;
      }
      ctx->host_times[2] += ms_since(tr);
      ++rounds;
      pending.clear();
    }
    const auto tw = std::chrono::steady_clock::now();
    CK(cudaEventSynchronize(gev[inflight.par]));
    ctx->host_times[1] += ms_since(tw);
    ctx->host_times[3] += 1.;
    const int nact_out = ctx->pinned[8 + 2 * inflight.par];
    const int64_t done_now = ctx->pinned[9 + 2 * inflight.par];
    unprocessed_bound -= inflight.issued;
    if (nact_out > inflight.nact_up || done_now > n || done_now < done_seen) {
      return fail(ctx, TMX_ERR_CUDA, "order loop: inconsistent done list");
    }
    for (int64_t j = done_seen; j < done_now; ++j) {
      const int32_t g = ctx->pinned_done[j];
      const int32_t ko = ctx->pinned_done[n + j];
      ctx->nmax_h[g] = ko;
      ctx->ngauss_h[g] = glf * ko;
      if (ctx->keep_valid) {
        ctx->keep_off_h[g] = ctx->pinned_keep[j];
      }
      ready.push_back(g);
    }
    done_seen = done_now;
    nact_known = nact_out;
    if (have_next) {
      // the queued group's bound can be tightened for the one after it
      next.nact_up = std::min(next.nact_up, nact_out);
      inflight = next;
    }
    have_inflight = have_next;
    if (nact_out > 0 && (int64_t)ready.size() >= round_min) {
      // at most round_max grains per round: a round's host set-up runs
      // while the GPU computes the next orders, and should not outlast them
      const size_t take = std::min<size_t>(ready.size(), (size_t)round_max);
      pending.assign(ready.begin(), ready.begin() + take);
      ready.erase(ready.begin(), ready.begin() + take);
      for (int32_t g : pending) {
        launched[g] = 1;
      }
    }
  }
  chain_range.reset();
  if ((rc = tl_mark(ctx, TMX_TL_LOOP_END, st))) {
    return rc;
  }

  // ---- per-grain outcome of the order loop
  CK(cudaMemcpyAsync(st0.data(), ctx->state.p, n * sizeof(TmxChainState),
                     cudaMemcpyDeviceToHost, st));
  if (ctx->keep_valid) {
    CK(cudaMemcpyAsync(ctx->pinned + 4, ctx->keep_ctl.p, 4 * sizeof(int32_t),
                       cudaMemcpyDeviceToHost, st));
  }
  {
    const auto tw = std::chrono::steady_clock::now();
    CK(cudaStreamSynchronize(st));
    ctx->host_times[1] += ms_since(tw);
  }
  if (ctx->keep_valid) {
    uint64_t used = 0;
    memcpy(&used, ctx->pinned + 6, sizeof(used));
    ctx->keep_used_last = (int64_t)used;
  }
  std::vector<int32_t> p2; // grains whose blocks have not been launched
  for (int64_t i = 0; i < n; ++i) {
    ctx->nmax_h[i] = st0[i].nmax;
    ctx->ngauss_h[i] = st0[i].ngauss;
    ctx->status_h[i] = st0[i].status | ctx->up_status[i];
    ctx->q_h[6 * i + 0] = st0[i].qsca;
    ctx->q_h[6 * i + 1] = st0[i].qext;
    ctx->q_h[6 * i + 4] = st0[i].dqs;
    ctx->q_h[6 * i + 5] = st0[i].dqe;
    if (st0[i].nmax > 0 && !launched[i]) {
      p2.push_back((int32_t)i);
    }
  }
  note_kmax(ctx);
  if (rounds == 0) {
    if ((rc = run_blocks(ctx, p2))) {
      return rc;
    }
    return tl_mark(ctx, TMX_TL_BATCH_END, st);
  }
  // the last round on this stream, then wait for the round streams
  if ((rc = run_blocks_round(ctx, p2, st, t_next, true, &t_next, true))) {
    return rc;
  }
  cudaEvent_t rounds_done;
  CK(cudaEventCreateWithFlags(&rounds_done, cudaEventDisableTiming));
  CK(cudaEventRecord(rounds_done, ctx->stream2));
  CK(cudaStreamWaitEvent(st, rounds_done, 0));
  CK(cudaEventRecord(rounds_done, ctx->stream3));
  CK(cudaStreamWaitEvent(st, rounds_done, 0));
  if (ctx->copy_stream) {
    CK(cudaEventRecord(rounds_done, ctx->copy_stream));
    CK(cudaStreamWaitEvent(st, rounds_done, 0));
  }
  CK(cudaEventDestroy(rounds_done));
  if ((rc = finish_blocks(ctx, t_next, rounds + 1))) {
    return rc;
  }
  if ((rc = tl_mark(ctx, TMX_TL_BATCH_END, st))) {
    return rc;
  }
  ctx->rounds_lu = true;
  return TMX_OK;
}

int tmx_tmatrix_batch(tmx_ctx *ctx, int64_t n, const double *r_ev,
                      const double *wavelength, const double *mr,
                      const double *mi, const double *axis_ratio,
                      const tmx_schedule *sched) {
  int rc = tmx_batch_upload(ctx, n, r_ev, wavelength, mr, mi, axis_ratio, sched);
  if (rc) {
    return rc;
  }
  return tmx_batch_compute(ctx);
}

int tmx_tmatrix_batch_fixed(tmx_ctx *ctx, int64_t n, const double *r_ev,
                            const double *wavelength, const double *mr,
                            const double *mi, const double *axis_ratio,
                            const int32_t *nmax, const int32_t *ngauss) {
  if (!ctx) {
    return TMX_ERR_INVALID;
  }
  if (n > 0 && (!nmax || !ngauss)) {
    return fail(ctx, TMX_ERR_INVALID, "null nmax/ngauss");
  }
  int32_t top = 2;
  for (int64_t i = 0; i < n; ++i) {
    if (nmax[i] < 1 || nmax[i] > TMX_MAX_NB || ngauss[i] < 1) {
      return fail(ctx, TMX_ERR_INVALID, "nmax must be in [1, 128], ngauss >= 1");
    }
    top = std::max(top, nmax[i]);
  }
  tmx_schedule S = {2, std::max(top + 1, 3), 1, 0, 1.e-4};
  int rc = tmx_batch_upload(ctx, n, r_ev, wavelength, mr, mi, axis_ratio, &S);
  if (rc) {
    return rc;
  }
  CK(cudaSetDevice(ctx->device));
  ctx->have_batch = false;
  ctx->lu_ready = false;
  if ((rc = tmx_release_rounds(ctx))) {
    return rc;
  }
  ctx->n = n;
  ++ctx->batch_seq;
  ctx->nmax_h.assign(n, 0);
  ctx->ngauss_h.assign(n, 0);
  ctx->status_h.assign(n, 0);
  ctx->q_h.assign(6 * n, 0.);
  ctx->t_off_h.assign(n, 0);
  ctx->flops_survey = 0.;
  std::vector<int32_t> p2;
  std::vector<int> ngs;
  for (int64_t i = 0; i < n; ++i) {
    ctx->status_h[i] = ctx->up_status[i];
    if (ctx->up_status[i] == 0) {
      ctx->nmax_h[i] = nmax[i];
      ctx->ngauss_h[i] = ngauss[i];
      p2.push_back((int32_t)i);
      ngs.push_back(ngauss[i]);
    }
  }
  if ((rc = ensure_gl(ctx, ngs))) {
    return rc;
  }
  CK(cudaMemsetAsync(ctx->status.p, 0, n * sizeof(int32_t), ctx->stream));
  if (n == 0) {
    ctx->p2_t_total = 0;
    ctx->have_batch = true;
    return TMX_OK;
  }
  return run_blocks(ctx, p2);
}

void *tmx_host_alloc(size_t bytes) {
  void *p = nullptr;
  if (bytes == 0 || cudaMallocHost(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void tmx_host_free(void *p) {
  if (p) {
    cudaFreeHost(p);
  }
}

int tmx_get_dispatch(const tmx_ctx *ctx, int32_t *family) {
  if (!ctx || !family) {
    return TMX_ERR_INVALID;
  }
  memcpy(family, ctx->dispatch, sizeof(ctx->dispatch));
  return TMX_OK;
}

int tmx_set_dispatch(tmx_ctx *ctx, const int32_t *family) {
  if (!ctx || !family) {
    return TMX_ERR_INVALID;
  }
  for (int b = 0; b < TMX_DISPATCH_BUCKETS; ++b) {
    if (family[b] < 0 || family[b] >= TMX_DISPATCH_FAMILIES ||
        tmx_block_family_capacity(family[b]) < kBucketTop[b]) {
      return fail(ctx, TMX_ERR_INVALID, "block family cannot run this size bucket");
    }
  }
  memcpy(ctx->dispatch, family, sizeof(ctx->dispatch));
  return TMX_OK;
}

static void drop_tune_events(tmx_ctx *ctx) {
  for (auto &e : ctx->tune_ev) {
    cudaEventDestroy(std::get<1>(e));
    cudaEventDestroy(std::get<2>(e));
  }
  ctx->tune_ev.clear();
}

int tmx_autotune(tmx_ctx *ctx, int64_t n, const double *r_ev,
                 const double *wavelength, const double *mr, const double *mi,
                 const double *axis_ratio, const int32_t *nmax,
                 const int32_t *ngauss, int reps, double *ms) {
  if (!ctx || n <= 0 || reps < 1) {
    return TMX_ERR_INVALID;
  }
  int32_t saved[TMX_DISPATCH_BUCKETS];
  memcpy(saved, ctx->dispatch, sizeof(saved));
  // per-batch milliseconds of each bucket under each family
  std::vector<double> t[TMX_DISPATCH_BUCKETS][TMX_DISPATCH_FAMILIES];
  int rc = TMX_OK;
  ctx->tuning = true;
  for (int f = 0; f < TMX_DISPATCH_FAMILIES && rc == TMX_OK; ++f) {
    // family f in every bucket it can run, the default elsewhere
    bool any = false;
    for (int b = 0; b < TMX_DISPATCH_BUCKETS; ++b) {
      const bool can = tmx_block_family_capacity(f) >= kBucketTop[b];
      ctx->dispatch[b] = can ? f : kDefaultDispatch[b];
      any = any || can;
    }
    if (!any) {
      continue;
    }
    // (a named range per family, so that a profiler can pick its launches)
    const std::string range_name = "tmx_autotune_" + std::string(kFamilyNames[f]);
    NvtxRange family_range(range_name.c_str());
    // one untimed batch, then reps timed ones
    for (int r = 0; r <= reps && rc == TMX_OK; ++r) {
      drop_tune_events(ctx);
      rc = tmx_tmatrix_batch_fixed(ctx, n, r_ev, wavelength, mr, mi, axis_ratio,
                                   nmax, ngauss);
      if (rc != TMX_OK) {
        break;
      }
      double sum[TMX_DISPATCH_BUCKETS] = {0.};
      bool seen[TMX_DISPATCH_BUCKETS] = {false};
      for (auto &e : ctx->tune_ev) {
        float x = 0.f;
        if (cudaEventSynchronize(std::get<2>(e)) != cudaSuccess ||
            cudaEventElapsedTime(&x, std::get<1>(e), std::get<2>(e)) != cudaSuccess) {
          rc = fail(ctx, TMX_ERR_CUDA, "autotune: event timing failed");
          break;
        }
        sum[std::get<0>(e)] += x;
        seen[std::get<0>(e)] = true;
      }
      for (int b = 0; b < TMX_DISPATCH_BUCKETS && r > 0; ++b) {
        if (seen[b] && ctx->dispatch[b] == f) {
          t[b][f].push_back(sum[b]);
        }
      }
    }
  }
  ctx->tuning = false;
  drop_tune_events(ctx);
  memcpy(ctx->dispatch, saved, sizeof(saved));
  if (rc != TMX_OK) {
    return rc;
  }
  // a bucket leaves its current family only for one at least kTuneMargin
  // faster: differences within timing noise keep the table as it was
  const double kTuneMargin = 0.05;
  for (int b = 0; b < TMX_DISPATCH_BUCKETS; ++b) {
    double med[TMX_DISPATCH_FAMILIES];
    int best = -1;
    for (int f = 0; f < TMX_DISPATCH_FAMILIES; ++f) {
      med[f] = -1.;
      std::vector<double> &v = t[b][f];
      if (!v.empty()) {
        std::sort(v.begin(), v.end());
        med[f] = (v.size() & 1) ? v[v.size() / 2]
                                : 0.5 * (v[v.size() / 2 - 1] + v[v.size() / 2]);
        if (best < 0 || med[f] < med[best]) {
          best = f;
        }
      }
      if (ms) {
        ms[b * TMX_DISPATCH_FAMILIES + f] = med[f];
      }
    }
    const int cur = saved[b];
    if (best >= 0 && best != cur &&
        (med[cur] < 0. || med[best] < (1. - kTuneMargin) * med[cur])) {
      ctx->dispatch[b] = best;
    }
  }
  return TMX_OK;
}

int tmx_batch_results(tmx_ctx *ctx, int32_t *nmax, int32_t *ngauss,
                      int32_t *status, double *q) {
  if (!ctx) {
    return TMX_ERR_INVALID;
  }
  if (!ctx->have_batch) {
    return fail(ctx, TMX_ERR_STATE, "no batch has been computed");
  }
  const size_t n = ctx->n;
  if (nmax) {
    memcpy(nmax, ctx->nmax_h.data(), n * sizeof(int32_t));
  }
  if (ngauss) {
    memcpy(ngauss, ctx->ngauss_h.data(), n * sizeof(int32_t));
  }
  if (status) {
    memcpy(status, ctx->status_h.data(), n * sizeof(int32_t));
  }
  if (q) {
    memcpy(q, ctx->q_h.data(), 6 * n * sizeof(double));
  }
  return TMX_OK;
}

int tmx_batch_tmatrix(tmx_ctx *ctx, int64_t grain, double *out) {
  if (!ctx || !out) {
    return TMX_ERR_INVALID;
  }
  if (!ctx->have_batch || grain < 0 || grain >= ctx->n) {
    return fail(ctx, TMX_ERR_STATE, "grain index out of range");
  }
  const int64_t sz = tmx_tmatrix_size(ctx->nmax_h[grain]);
  if (sz == 0) {
    return TMX_OK;
  }
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(out, (const cplx *)ctx->T.p + ctx->t_off_h[grain],
                     sz * sizeof(cplx), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return TMX_OK;
}

int tmx_batch_tmatrix_total(tmx_ctx *ctx, int64_t *total) {
  if (!ctx || !total) {
    return TMX_ERR_INVALID;
  }
  if (!ctx->have_batch) {
    return fail(ctx, TMX_ERR_STATE, "no batch has been computed");
  }
  *total = ctx->p2_t_total;
  return TMX_OK;
}

int tmx_batch_tmatrices(tmx_ctx *ctx, double *out, int64_t *offsets) {
  if (!ctx || (!out && !offsets)) {
    return TMX_ERR_INVALID;
  }
  if (!ctx->have_batch) {
    return fail(ctx, TMX_ERR_STATE, "no batch has been computed");
  }
  CK(cudaSetDevice(ctx->device));
  if (offsets) {
    for (int64_t i = 0; i < ctx->n; ++i) {
      offsets[i] = (ctx->nmax_h[i] > 0) ? ctx->t_off_h[i] : -1;
    }
  }
  const int64_t total = ctx->p2_t_total;
  if (out && total > 0) {
    // into the sink only what the block rounds have not streamed already
    const int64_t from = (out == ctx->sink) ? std::min(ctx->sink_done, total) : 0;
    if (from < total) {
      CK(cudaMemcpyAsync(out + 2 * from, (const cplx *)ctx->T.p + from,
                         (total - from) * sizeof(cplx), cudaMemcpyDeviceToHost,
                         ctx->stream));
    }
    // the streamed copies ran on the round streams, which ctx->stream
    // joined at the end of the batch
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return TMX_OK;
}

int tmx_set_tmatrix_sink(tmx_ctx *ctx, double *host, int64_t capacity) {
  if (!ctx || capacity < 0 || (capacity > 0 && !host)) {
    return TMX_ERR_INVALID;
  }
  if (host) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, host) != cudaSuccess ||
        at.type != cudaMemoryTypeHost) {
      cudaGetLastError();
      return fail(ctx, TMX_ERR_INVALID,
                  "the T-matrix sink must be page-locked host memory "
                  "(tmx_host_alloc or cudaHostRegister)");
    }
  }
  // copies into the previous sink must be complete before it is released
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream2));
  CK(cudaStreamSynchronize(ctx->stream3));
  if (ctx->copy_stream) {
    CK(cudaStreamSynchronize(ctx->copy_stream));
  }
  ctx->sink = host;
  ctx->sink_cap = host ? capacity : 0;
  ctx->sink_done = 0;
  return TMX_OK;
}

int tmx_timer_start(tmx_ctx *ctx) {
  if (!ctx) {
    return TMX_ERR_INVALID;
  }
  CK(cudaSetDevice(ctx->device));
  if (!ctx->t0) {
    CK(cudaEventCreate(&ctx->t0));
    CK(cudaEventCreate(&ctx->t1));
  }
  CK(cudaEventRecord(ctx->t0, ctx->stream));
  return TMX_OK;
}

int tmx_timer_stop(tmx_ctx *ctx, double *ms) {
  if (!ctx || !ms || !ctx->t0) {
    return TMX_ERR_INVALID;
  }
  CK(cudaEventRecord(ctx->t1, ctx->stream));
  CK(cudaEventSynchronize(ctx->t1));
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, ctx->t0, ctx->t1));
  *ms = f;
  return TMX_OK;
}

int tmx_profile_enable(tmx_ctx *ctx, int on) {
  if (!ctx) {
    return TMX_ERR_INVALID;
  }
  CK(cudaSetDevice(ctx->device));
  CK(cudaDeviceSynchronize());
  for (auto &p : ctx->prof) {
    p.pending.clear();
    p.ms = 0.;
    p.launches = 0;
    p.flops = 0.;
    p.bytes = 0.;
  }
  ctx->prof_used = 0;
  ctx->tl_pending.clear();
  ctx->tl_done.clear();
  ctx->profiling = on != 0;
  if (ctx->profiling) {
    if (!ctx->tl_origin) {
      CK(cudaEventCreate(&ctx->tl_origin));
    }
    CK(cudaEventRecord(ctx->tl_origin, ctx->stream));
  }
  // events for a few batches, made before any timed work
  while (ctx->profiling && ctx->prof_pool.size() < 2048) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    ctx->prof_pool.push_back(e);
  }
  return TMX_OK;
}

int tmx_profile_bytes(tmx_ctx *ctx, int kernel, double *bytes) {
  if (!ctx || !bytes || kernel < 0 || kernel >= TMX_PROF_KERNELS) {
    return TMX_ERR_INVALID;
  }
  *bytes = ctx->prof[kernel].bytes;
  return TMX_OK;
}

int tmx_batch_host_times(tmx_ctx *ctx, double *out) {
  if (!ctx || !out) {
    return TMX_ERR_INVALID;
  }
  for (int i = 0; i < 4; ++i) {
    out[i] = ctx->host_times[i];
  }
  return TMX_OK;
}

int tmx_profile_timeline(tmx_ctx *ctx, int64_t cap, double *records,
                         int64_t *count) {
  if (!ctx || cap < 0 || (cap > 0 && !records) || !count) {
    return TMX_ERR_INVALID;
  }
  CK(cudaSetDevice(ctx->device));
  CK(cudaDeviceSynchronize());
  if (ctx->profiling || !ctx->tl_pending.empty()) {
    const int rc = prof_resolve(ctx);
    if (rc) {
      return rc;
    }
  }
  const int64_t nrec = (int64_t)ctx->tl_done.size() / 5;
  *count = nrec;
  if (cap > 0) {
    memcpy(records, ctx->tl_done.data(),
           (size_t)std::min(cap, nrec) * 5 * sizeof(double));
  }
  return TMX_OK;
}

int tmx_profile_read(tmx_ctx *ctx, int kernel, double *ms, int64_t *launches,
                     double *flops) {
  if (!ctx || kernel < 0 || kernel >= TMX_PROF_KERNELS) {
    return TMX_ERR_INVALID;
  }
  CK(cudaSetDevice(ctx->device));
  CK(cudaDeviceSynchronize());
  const int rc = prof_resolve(ctx);
  if (rc) {
    return rc;
  }
  if (ms) {
    *ms = ctx->prof[kernel].ms;
  }
  if (launches) {
    *launches = ctx->prof[kernel].launches;
  }
  if (flops) {
    *flops = ctx->prof[kernel].flops;
  }
  return TMX_OK;
}

double tmx_batch_flops_survey(const tmx_ctx *ctx) {
  return ctx ? ctx->flops_survey : 0.;
}

int tmx_probe_fp64(tmx_ctx *ctx, int kind, double *tflops) {
  if (!ctx || !tflops) {
    return TMX_ERR_INVALID;
  }
  CK(cudaSetDevice(ctx->device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  const int blocks = sms * 8;
  const int iters = 4096;
  int rc;
  if ((rc = ensure(ctx, ctx->probe, (size_t)blocks * 256 * sizeof(double)))) {
    return rc;
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    CK(cudaEventRecord(e0, ctx->stream));
    if (kind == 0) {
      tmx_launch_probe_dfma((double *)ctx->probe.p, iters, blocks, ctx->stream);
    } else {
      tmx_launch_probe_dmma((double *)ctx->probe.p, iters, blocks, ctx->stream);
    }
    LAUNCHED();
    CK(cudaEventRecord(e1, ctx->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0) {
      best = std::min(best, ms);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  double flops;
  if (kind == 0) {
    flops = 2.0 * 8 * iters * (double)blocks * 256;
  } else {
    flops = 512.0 * 8 * iters * (double)blocks * (256 / 32);
  }
  *tflops = flops / (best * 1e-3) / 1e12;
  return TMX_OK;
}

} // extern "C"

// ------------------------------------------- helpers for other host units --

int tmx_ensure_gl(tmx_ctx *ctx, const std::vector<int> &ngs) {
  return ensure_gl(ctx, ngs);
}

int tmx_ensure_wigner(tmx_ctx *ctx, const std::vector<std::pair<int, int>> &keys,
                      bool all_m, std::vector<int> &set_ids) {
  return ensure_wigner(ctx, keys, all_m, set_ids);
}

int tmx_run_blocks(tmx_ctx *ctx, const std::vector<int32_t> &grains) {
  return run_blocks(ctx, grains);
}
