// Internal: the context object shared by the host-side translation units.
#pragma once

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <array>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/tmx.h"
#include "tmx_common.cuh"
#include "tmx_kernels.h"

namespace {

// NVTX range for the duration of a scope (phase markers for profilers)
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
};

} // namespace

struct tmx_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;  // every launch unless noted (high priority)
  cudaStream_t stream2 = nullptr; // blocks of grains that converged while the
  cudaStream_t stream3 = nullptr; // order loop continues (low priority);
                                  // rounds alternate between the two, so a
                                  // round starts while the previous drains
  cudaStream_t aux[6] = {};       // further class-size buckets of a block
                                  // round: [0, 1] beside stream, [2, 3]
                                  // beside stream2, [4, 5] beside stream3
  cudaMemPool_t pool = nullptr;   // device memory of this context; keeps
                                  // freed blocks for reuse (no release)
  std::string err;
  int64_t launches = 0;
  // Gauss-Legendre cache: lower-half nodes of the 2 * ngauss rule
  std::vector<int64_t> gl_off_h;
  std::vector<double> gl_x_h, gl_w_h;
  DevBuf gl_x, gl_w, gl_off;
  bool gl_dirty = true;
  // Wigner d table sets, keyed by (nmax, ngauss, all m?)
  std::map<std::tuple<int, int, int>, int> wig_sets;
  std::vector<int64_t> wig_off_h;
  int64_t wig_used = 0;
  DevBuf wig, wig_off;
  // batch buffers
  DevBuf grains, state, state0, act0, act1, actinit, count, slots, items, tab,
      nsc, scratch, diag, T, q, status, probe;
  // uploaded batch (device-resident inputs)
  bool uploaded = false;
  int64_t up_n = 0;
  int up_nact = 0;
  tmx_schedule up_sched;
  std::vector<int32_t> up_status;
  std::vector<TmxGrain> up_grains;
  // observables (get_table): cached Clebsch-Gordan table and work buffers
  DevBuf cg, cg_off;
  int cg_nmax = 0;
  DevBuf Ta, o_angles, o_phis, o_wts, o_coef, o_shw, o_og, o_work, o_sj, o_qj,
      o_S, o_gq, o_gz, o_cq, o_cz, o_pairs, o_grp, o_x;
  // plan of the observable kernels (first pair of each grain, job groups)
  int64_t o_ngrains = 0, o_npairs = 0;
  int o_nbmax = 1, o_ngrp = 0;
  // orientation-average work order: pair-major item starts (o_pairs, pmax^2
  // + 1) and the grains by descending order (o_ord)
  DevBuf o_ord;
  int o_pmax = 1;
  // angles of the current plan (o_angles) and their pi / tau columns
  int o_nangles = 0;
  DevBuf o_wcol;
  // flops of one matrix set in the orientation average and the amplitudes
  // of the current plan (counted while profiling)
  double o_fl_orient = 0., o_fl_amp = 0.;
  int32_t *pinned = nullptr;     // 16 words: [4..7] the table arena's
                                 // counters, [8 + 2 p] / [9 + 2 p] list and
                                 // done-list lengths after an order group of
                                 // parity p, [12] the first list's length
  DevBuf done;                    // grains whose order became final, in order
  int32_t *pinned_done = nullptr; // host copy of new done-list entries
  int64_t pinned_done_cap = 0;
  // timing: events on the library stream
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  bool profiling = false;
  struct Prof {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
    double ms = 0.;
    int64_t launches = 0;
    double flops = 0.;
    double bytes = 0.; // algorithmic bytes (each operand read or written once)
  } prof[TMX_PROF_KERNELS]; // tmx_profile_kernel
  // timing events, reused once their pairs are resolved (at the next read of
  // the profile), so that a profiled batch creates none
  std::vector<cudaEvent_t> prof_pool;
  size_t prof_used = 0;
  // timeline of the profiled launches (tmx_profile_timeline): kind, stream
  // and launch size with the events around the launch, resolved to ms after
  // tl_origin (recorded by tmx_profile_enable on the library stream)
  struct TlRec {
    int32_t kind, stream, info;
    cudaEvent_t a, b;
  };
  std::vector<TlRec> tl_pending;
  std::vector<double> tl_done; // 5 per record: kind, stream, info, start, end
  cudaEvent_t tl_origin = nullptr;
  // Block rounds of the last tmx_batch_compute, kept for the gradients: each
  // round's tables, slot and item lists and LU factors (pool allocations
  // released when the next batch starts). rounds_lu: they cover every grain
  // of the batch, so the gradients need no second pass of the blocks.
  struct RoundRec {
    double *tab = nullptr, *nsc = nullptr;
    bool own_tables = true; // false: tab and nsc are the batch's table arena
    bool borrowed = false;  // slots, items and lu are context buffers
    TmxSlot *slots = nullptr;
    TmxItem *items = nullptr;
    cplx *lu = nullptr;
    std::vector<int> nb; // class size per item (descending)
    // or, for a device-driven batch: per size bucket, largest first, the
    // item range [i0, i1) and an upper bound of its class sizes
    std::vector<std::array<int64_t, 3>> seg;
    int64_t scr_total = 0;
  };
  std::vector<RoundRec> rounds_kept;
  bool keep_rounds = false;
  bool rounds_lu = false;
  // block-kernel family per size bucket (tmx_set_dispatch, tmx_autotune)
  int32_t dispatch[TMX_DISPATCH_BUCKETS] = {0, 1, 2, 3, 4};
  // autotuning: bucket launches serialised on the round's stream and timed
  // (bucket, start, end)
  bool tuning = false;
  std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> tune_ev;
  std::vector<double> survey_cache; // survey-model flops per order, this glf
  int survey_glf = 0, survey_min = 0;
  double flops_survey = 0.; // survey-model flops of the last batch
  // last batch
  int64_t n = 0;
  bool have_batch = false;
  bool t_averaged = false; // T holds orientation averages (no gradients)
  // generation counters: batch_seq changes whenever the batch's grains,
  // orders, T-matrix offsets or T-matrices change, plan_seq at every upload
  // of an observable plan; obs_key identifies the plan of the last
  // batch_observable_setup (reused while both counters and its angles and
  // coefficients are unchanged)
  uint64_t batch_seq = 0, plan_seq = 0;
  // device-driven batch (tmx_graph.cu): mode, buffers, the executable graph
  // and the key (sizes and addresses) it was built for, and the T-matrix /
  // LU storage hints grown by a batch that outgrew them
  int batch_mode = TMX_BATCH_HOST, last_mode = TMX_BATCH_HOST;
  DevBuf gm_state, gm_iter, gm_tab, gm_nsc, gm_scr, gm_diag, gm_slots, gm_items,
      gm_rslots, gm_bitems, gm_bptr, gm_bcap, gm_tpl, gm_tpl_off, gm_full,
      gm_tsize, gm_toff, gm_lu, gm_luscr, gm_allitems, gm_steps;
  cudaGraph_t gm_graph = nullptr;
  cudaGraphExec_t gm_exec = nullptr;
  std::vector<uint64_t> gm_key;
  cudaStream_t gm_cs = nullptr, gm_rs = nullptr, gm_bs[TMX_GM_BUCKETS] = {};
  int64_t gm_t_hint = 0, gm_lu_hint = 0;
  int64_t gm_last_t = 0;
  int gm_counts[2] = {0, 0};       // the last graph batch's order steps and rounds
  // largest final order of the last batch and its schedule (min order, last
  // order, Gauss-Legendre factor, tolerance): the device-driven graph's extent
  int kmax_seen = 0;
  int kmax_sched[3] = {0, 0, 0};
  double kmax_tol = -1.;
  // the last graph's extent (last order) and its schedule
  int gm_kg = 0;
  int gm_kg_sched[3] = {0, 0, 0};
  double gm_kg_tol = -1.;
  // host-side times of the last tmx_batch_compute (ms): wall time, time
  // blocked on the order loop's events and the final synchronisation, host
  // set-up of block rounds, and the number of order groups
  double host_times[4] = {0., 0., 0., 0.};
  struct ObsKey {
    bool valid = false;
    uint64_t batch_seq = 0, plan_seq = 0;
    std::vector<double> thetas, coeffs;
    bool has_coeffs = false;
  } obs_key;
  // o_S holds the amplitudes of the batch's T-matrices under the plan of
  // obs_key (tmx_batch_observables); the gradients of the same plan reuse them
  bool obs_s_valid = false;
  std::vector<int32_t> nmax_h, ngauss_h, status_h;
  std::vector<double> q_h;
  std::vector<int64_t> t_off_h;
  // block schedule of the last batch (phase 2), reused by the tangents; its
  // tables, slots, items and scratch live in the p2 buffers. p2_rounds > 1:
  // the blocks ran in two rounds and the buffers hold the last round only.
  DevBuf p2tab, p2nsc, p2scratch, p2slots, p2items;
  int p2_rounds = 0;
  std::vector<TmxSlot> p2_slots;
  std::vector<TmxItem> p2_items;
  bool lu_ready = false; // ctx->lu holds the LU factors of every p2 item
  std::vector<int> p2_nb;
  // block items of one grain of order N, in (m, class) order: m << 8 | cls
  // and the class size; and the (size, count) bins of that list
  struct ItemTemplate {
    std::vector<int32_t> mc, nb;
    std::vector<std::pair<int32_t, int32_t>> bins;
    // flops of the grain's items: fl_a * ngauss + fl_b (item_flops)
    double fl_a = 0., fl_b = 0.;
  };
  std::vector<ItemTemplate> item_tpl; // indexed by N
  int64_t p2_scr_total = 0, p2_t_total = 0;
  DevBuf lu, dT, tscr, dTa, dS; // tangent buffers
  int o_nsj = 0, o_nqj = 0;     // per-grain observable job counts
  // events that order a free on `stream` after the work queued so far on the
  // round streams, their bucket streams (stream2, stream3, aux[0..5]) and
  // the copy stream
  cudaEvent_t drain_ev[9] = {};
  // device-to-host copies of streamed T-matrices (created with the first
  // sink copy): a round's copy waits for the round, the rounds that follow
  // on the same round stream do not wait for the copy
  cudaStream_t copy_stream = nullptr;
  // page-locked host destination of the T-matrices (tmx_set_tmatrix_sink):
  // every block round copies its T range there as soon as its blocks are
  // done; sink_done = complex elements [0, sink_done) already copied for the
  // current batch
  double *sink = nullptr;
  int64_t sink_cap = 0;
  int64_t sink_done = 0;
  // final-order tables of the grains of a batched computation, copied out of
  // the order loop's buffers as the grains become final (k_keep_tables):
  // arena, per-grain offsets (device and host, -1: none), per done-list
  // entry offsets, done-list positions, and the copy kernel's counters
  // ({next entry, ticket, doubles used})
  DevBuf keep_arena, keep_tab, keep_q, done_pos, keep_ctl;
  std::vector<int64_t> keep_off_h;
  int64_t *pinned_keep = nullptr;
  int64_t pinned_keep_cap = 0;
  bool keep_valid = false;
  int64_t keep_used_last = 0; // doubles the last batch used
};

#define CK(call)                                                               \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);           \
      return TMX_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)

#define LAUNCHED()                                                             \
  do {                                                                         \
    ++ctx->launches;                                                           \
    CK(cudaGetLastError());                                                    \
  } while (0)

// Makes ctx->stream wait for everything queued so far on the other streams
// of the context. Every free of a shared buffer (Wigner and quadrature
// tables, T, the Q sums) is issued on ctx->stream while block rounds may
// still run on the round streams and read it; the pool may hand a freed
// block to the next allocation as soon as the free is complete in stream
// order, so the free must come after those readers.
static inline int order_after_rounds(tmx_ctx *ctx) {
  cudaStream_t others[9] = {ctx->stream2, ctx->stream3, ctx->aux[0], ctx->aux[1],
                            ctx->aux[2],  ctx->aux[3],  ctx->aux[4], ctx->aux[5],
                            ctx->copy_stream};
  for (int i = 0; i < 9; ++i) {
    if (!others[i]) {
      continue;
    }
    if (!ctx->drain_ev[i]) {
      CK(cudaEventCreateWithFlags(&ctx->drain_ev[i], cudaEventDisableTiming));
    }
    CK(cudaEventRecord(ctx->drain_ev[i], others[i]));
    CK(cudaStreamWaitEvent(ctx->stream, ctx->drain_ev[i], 0));
  }
  return TMX_OK;
}

// executed flops of one class item: assembly (4 real FMAs per entry, node
// and term; 2 terms for m = 0), LU (8/3 nb^3) and the two triangular solves
// with nb right-hand sides (8 nb^3)
static inline double item_flops(int nb, int m, int ng) {
  const double b = nb;
  const double terms = (m == 0) ? 2. : 4.;
  return 8. * terms * b * b * ng + (8. / 3.) * b * b * b + 8. * b * b * b;
}

// dispatch bucket of a launch whose largest class has nb members, and the
// family the context's table names for it
static inline int dispatch_bucket(int nb) {
  return (nb <= 8) ? 0 : (nb <= 16) ? 1 : (nb <= 32) ? 2 : (nb <= 64) ? 3 : 4;
}
static inline int dispatch_family(const tmx_ctx *ctx, int max_nb) {
  return ctx->dispatch[dispatch_bucket(max_nb)];
}

static inline int prof_event(tmx_ctx *ctx, cudaEvent_t *e) {
  if (ctx->prof_used == ctx->prof_pool.size()) {
    cudaEvent_t n;
    CK(cudaEventCreate(&n));
    ctx->prof_pool.push_back(n);
  }
  *e = ctx->prof_pool[ctx->prof_used++];
  return 0;
}

static inline int prof_begin(tmx_ctx *ctx, int k, cudaEvent_t *a,
                             cudaStream_t st = nullptr) {
  if (!ctx->profiling) {
    return 0;
  }
  int rc = prof_event(ctx, a);
  if (rc) {
    return rc;
  }
  CK(cudaEventRecord(*a, st ? st : ctx->stream));
  (void)k;
  return 0;
}

// index of a context stream in the timeline: 0 library stream, 1 and 2 the
// round streams, 3..8 the bucket streams, -1 any other
static inline int stream_index(const tmx_ctx *ctx, cudaStream_t st) {
  if (!st || st == ctx->stream) {
    return 0;
  }
  if (st == ctx->stream2) {
    return 1;
  }
  if (st == ctx->stream3) {
    return 2;
  }
  for (int i = 0; i < 6; ++i) {
    if (st == ctx->aux[i]) {
      return 3 + i;
    }
  }
  return -1;
}

// a point on the timeline (kind < 0: TMX_TL_* marks)
static inline int tl_mark(tmx_ctx *ctx, int kind, cudaStream_t st) {
  if (!ctx->profiling) {
    return 0;
  }
  cudaEvent_t a;
  int rc = prof_event(ctx, &a);
  if (rc) {
    return rc;
  }
  CK(cudaEventRecord(a, st ? st : ctx->stream));
  ctx->tl_pending.push_back({kind, stream_index(ctx, st), 0, a, a});
  return 0;
}

// info: the launch's work items (timeline only)
static inline int prof_end(tmx_ctx *ctx, int k, cudaEvent_t a, double flops,
                           cudaStream_t st = nullptr, double bytes = 0.,
                           int info = 0) {
  if (!ctx->profiling) {
    return 0;
  }
  cudaEvent_t b;
  int rc = prof_event(ctx, &b);
  if (rc) {
    return rc;
  }
  CK(cudaEventRecord(b, st ? st : ctx->stream));
  ctx->tl_pending.push_back({k, stream_index(ctx, st), info, a, b});
  ctx->prof[k].pending.push_back({a, b});
  ctx->prof[k].launches += 1;
  ctx->prof[k].flops += flops;
  ctx->prof[k].bytes += bytes;
  return 0;
}

// resolve recorded event pairs (after every stream has finished them) and
// return their events to the pool
static inline int prof_resolve(tmx_ctx *ctx) {
  for (auto &p : ctx->prof) {
    for (auto &e : p.pending) {
      float ms = 0.f;
      CK(cudaEventSynchronize(e.second));
      CK(cudaEventElapsedTime(&ms, e.first, e.second));
      p.ms += ms;
    }
    p.pending.clear();
  }
  for (const auto &r : ctx->tl_pending) {
    float t0 = 0.f, t1 = 0.f;
    CK(cudaEventSynchronize(r.b));
    CK(cudaEventElapsedTime(&t0, ctx->tl_origin, r.a));
    CK(cudaEventElapsedTime(&t1, ctx->tl_origin, r.b));
    const double v[5] = {(double)r.kind, (double)r.stream, (double)r.info,
                         (double)t0, (double)t1};
    ctx->tl_done.insert(ctx->tl_done.end(), v, v + 5);
  }
  ctx->tl_pending.clear();
  ctx->prof_used = 0;
  return 0;
}

static inline int fail(tmx_ctx *ctx, int code, const std::string &msg) {
  if (ctx) {
    ctx->err = msg;
  }
  return code;
}

// grow-only device buffer; contents are not preserved
static inline int ensure(tmx_ctx *ctx, DevBuf &b, size_t bytes) {
  if (bytes == 0) {
    bytes = 16;
  }
  if (b.cap >= bytes) {
    return TMX_OK;
  }
  // a reallocated buffer has lost its contents: no cached observable plan
  // may be reused after this
  ++ctx->plan_seq;
  if (b.p) {
    int rc = order_after_rounds(ctx);
    if (rc) {
      return rc;
    }
    CK(cudaFreeAsync(b.p, ctx->stream));
    b.p = nullptr;
    b.cap = 0;
  }
  size_t want = bytes + bytes / 4;
  cudaError_t e = cudaMallocFromPoolAsync(&b.p, want, ctx->pool, ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    e = cudaMallocFromPoolAsync(&b.p, bytes, ctx->pool, ctx->stream);
    want = bytes;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, TMX_ERR_NOMEM,
                "device allocation of " + std::to_string(bytes) + " bytes failed");
  }
  b.cap = want;
  return TMX_OK;
}

// grow-only device buffer that keeps its first `keep` bytes
static inline int ensure_keep(tmx_ctx *ctx, DevBuf &b, size_t bytes, size_t keep) {
  if (b.cap >= bytes) {
    return TMX_OK;
  }
  DevBuf nb;
  size_t want = std::max(bytes, b.cap * 2);
  if (cudaMallocFromPoolAsync(&nb.p, want, ctx->pool, ctx->stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, TMX_ERR_NOMEM, "device allocation failed (table cache)");
  }
  nb.cap = want;
  if (b.p) {
    int rc = order_after_rounds(ctx);
    if (rc) {
      return rc;
    }
    if (keep) {
      CK(cudaMemcpyAsync(nb.p, b.p, keep, cudaMemcpyDeviceToDevice,
                         ctx->stream));
    }
    CK(cudaFreeAsync(b.p, ctx->stream));
  }
  b = nb;
  return TMX_OK;
}

// Clebsch-Gordan table for all (n1, n2) <= nmax (tmx_table.cu)
int tmx_ensure_cg(tmx_ctx *ctx, int nmax);

// Host helpers of tmx_host.cu shared with the other host units: quadrature
// and Wigner table caches, and every block of the given grains at their
// orders in ctx->nmax_h / ctx->ngauss_h (one round, then the Q sums).
#define TMX_HIDDEN __attribute__((visibility("hidden")))
TMX_HIDDEN int tmx_ensure_gl(tmx_ctx *ctx, const std::vector<int> &ngs);
TMX_HIDDEN int tmx_ensure_wigner(tmx_ctx *ctx,
                                 const std::vector<std::pair<int, int>> &keys,
                                 bool all_m, std::vector<int> &set_ids);
TMX_HIDDEN int tmx_run_blocks(tmx_ctx *ctx, const std::vector<int32_t> &grains);

// Blocks of the last batch again in one round (tmx_host.cu), so that the p2
// buffers hold the whole schedule for the tangent kernels.
extern "C" __attribute__((visibility("hidden"))) int tmx_rerun_blocks(tmx_ctx *ctx);
extern "C" __attribute__((visibility("hidden"))) int tmx_release_rounds(tmx_ctx *ctx);
