// Device-driven batch (TMX_BATCH_GRAPH): the order loop and the block rounds
// of tmx_batch_compute as one CUDA graph whose conditional WHILE node runs
// on the GPU until no grain is left, so the host uploads the batch's
// descriptors, launches the graph once and reads the results.
//
// Reference semantics are those of the host-driven loop (TaskManager.hpp:
// 1146-1197 chain of TMatrixM0Task per order, :1313-1327 TMatrixMAllTask
// once the order is final): every order step of every active grain, the
// convergence test in the reference's order, and the blocks of every m at
// the final order. One iteration of the WHILE body is one order k:
//   k_gm_begin      iteration parameters (order, m = 0 Wigner set, table
//                   strides, size bucket of the m = 0 classes) and the item
//                   ranges of the round formed below
//   k_gm_prep       slots and m = 0 items of the active list
//   k_tables        node scalars and Bessel tables of the active grains
//   block kernels   the m = 0 classes (one launch per size bucket, gated)
//   k_converge      sums, test, next active list, done list
//   k_keep_tables   final-order tables of the grains that became final
// and, beside them (a second branch of the body), the round of the grains
// that became final in the previous iteration:
//   k_gm_round      slots and items of those grains (every m and class, into
//                   per-size-bucket item arrays), T-matrix and LU offsets
//   k_gm_round_mid  the round's item and slot ranges
//   block kernels   one launch per size bucket, on the round's ranges
//   k_qsums         Q sums of the round's grains
// then k_gm_swap / k_gm_end: the next active list becomes the current one,
// the order advances, and the WHILE condition is set to whether a grain is
// still active or a round is pending.
//
// Buffers are sized before the graph is built (no allocation inside):
// tables for every grain at the largest order, the arena for every grain's
// final-order tables, and T-matrix and LU storage from an estimate; a batch
// that outgrows the estimate is flagged on the device and the host computes
// it again with the host-driven loop (and a larger estimate next time).
#include <algorithm>
#include <vector>

#include "tmx_ctx.h"

// ------------------------------------------------------------- kernels --

__global__ void k_gm_begin(TmxGState *G, TmxGIter *I, const int32_t *__restrict__ m0_sets,
                           int min_order, int glf) {
  if (threadIdx.x != 0 || blockIdx.x != 0) {
    return;
  }
  const int k = G->k;
  TmxGIter it;
  it.order = k;
  it.ngauss = glf * k;
  it.wig_n = m0_sets[min(k, G->last_order) - min_order];
  const int cm = (k + 1) / 2;
  it.bucket = (cm <= 8) ? 0 : (cm <= 16) ? 1 : (cm <= 32) ? 2 : (cm <= 64) ? 3 : 4;
  TmxChainBase &b = it.base;
  b.slot = 0;
  b.tab = b.nsc = b.diag = b.scr = 0;
  b.tab_stride = (int64_t)glf * k * k * TMX_NQ;
  b.nsc_stride = (int64_t)glf * k * TMX_NS;
  b.diag_stride = 2 * (int64_t)k;
  b.scr_stride = 2 * (int64_t)cm * cm;
  *I = it;
  // the next active list starts empty; the round of this iteration covers
  // the done entries [round_lo, round_hi) fixed by the previous iteration
  G->cnt[2] = 0;
  for (int q = 0; q < TMX_GM_BUCKETS; ++q) {
    G->rng[q][0] = G->fill[q];
    G->rng[q][1] = G->fill[q];
  }
  G->srng[0] = G->nslots;
  G->srng[1] = G->nslots;
}

// slots and m = 0 items of every active position p < n (positions at or past
// the list's length get an empty slot: order 0, no classes, no nodes)
__global__ void k_gm_prep(const TmxGState *__restrict__ G, const TmxGIter *__restrict__ I,
                          const int32_t *__restrict__ active, int n, TmxSlot *slots,
                          TmxItem *items) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) {
    return;
  }
  const TmxGIter it = *I;
  const bool valid = p < G->cnt[0];
  TmxSlot s;
  s.grain = valid ? active[p] : 0;
  s.nmax = valid ? it.order : 0;
  s.ngauss = valid ? it.ngauss : 0;
  s.wig_n = it.wig_n;
  s.tab = p * it.base.tab_stride;
  s.nsc = p * it.base.nsc_stride;
  s.tout = -1;
  s.diag = p * it.base.diag_stride;
  slots[p] = s;
  for (int c = 0; c < 4; ++c) {
    TmxItem t;
    t.slot = p;
    t.m = 0;
    t.cls = (int16_t)c;
    t.scratch = (4 * (int64_t)p + c) * it.base.scr_stride;
    items[4 * p + c] = t;
  }
}

// The round: one thread per done entry of [round_lo, round_hi). A grain's
// items come from the template of its order (tpl_off[N] .. tpl_off[N + 1]
// in tpl, (m << 8 | class) and the class size), into the item array of
// their size bucket; its T-matrix and each item's LU factors get offsets
// from bump counters. A grain without kept tables or beyond the T / LU
// capacity sets the overflow flag (the host then recomputes the batch).
__global__ void k_gm_round(TmxGState *G, const int32_t *__restrict__ done_list,
                           const int32_t *__restrict__ done_ord,
                           const int64_t *__restrict__ keep_tab,
                           const int32_t *__restrict__ tpl_off,
                           const int32_t *__restrict__ tpl,
                           const int32_t *__restrict__ full_sets,
                           const int64_t *__restrict__ tsize, int glf, int min_order,
                           TmxSlot *rslots, int nslot_cap, TmxItem *const *bitems,
                           const int32_t *__restrict__ bcap, int64_t *t_off,
                           unsigned long long t_cap, unsigned long long lu_cap) {
  const int q = G->round_lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G->round_hi) {
    return;
  }
  const int g = done_list[q];
  const int N = done_ord[q];
  const int64_t tab = keep_tab[g];
  const int64_t ts = tsize[N];
  if (tab < 0) {
    atomicOr(&G->overflow, 1);
    return;
  }
  const int s = atomicAdd(&G->nslots, 1);
  if (s >= nslot_cap) {
    atomicOr(&G->overflow, 2);
    return;
  }
  const unsigned long long toff = atomicAdd(&G->t_used, (unsigned long long)ts);
  // the LU factors of the grain's items, one bump for all of them
  unsigned long long lu_need = 0;
  for (int j = tpl_off[N]; j < tpl_off[N + 1]; ++j) {
    const int nb = tpl[2 * j + 1];
    lu_need += 2ull * nb * nb;
  }
  const unsigned long long lu0 = atomicAdd(&G->lu_used, lu_need);
  if (toff + ts > t_cap || lu0 + lu_need > lu_cap) {
    // out of storage: the slot stays empty (order 0: the Q sums skip it) and
    // the host computes the batch again
    atomicOr(&G->overflow, 4);
    TmxSlot e = {};
    e.grain = g;
    rslots[s] = e;
    return;
  }
  TmxSlot sl;
  sl.grain = g;
  sl.nmax = N;
  sl.ngauss = glf * N;
  sl.wig_n = full_sets[N - min_order];
  sl.tab = tab;
  // (k_keep_tables puts the node scalars at the next multiple of 16)
  sl.nsc = tab + (((int64_t)sl.ngauss * N * TMX_NQ + 15) & ~(int64_t)15);
  sl.tout = (int64_t)toff;
  sl.diag = 0;
  rslots[s] = sl;
  t_off[g] = (int64_t)toff;
  unsigned long long lu = lu0;
  for (int j = tpl_off[N]; j < tpl_off[N + 1]; ++j) {
    const int mc = tpl[2 * j];
    const int nb = tpl[2 * j + 1];
    const int b = (nb <= 8) ? 0 : (nb <= 16) ? 1 : (nb <= 32) ? 2 : (nb <= 64) ? 3 : 4;
    const int pos = atomicAdd(&G->fill[b], 1);
    if (pos >= bcap[b]) {
      atomicOr(&G->overflow, 8);
      return;
    }
    TmxItem t;
    t.slot = s;
    t.m = (int16_t)(mc >> 8);
    t.cls = (int16_t)(mc & 0xff);
    t.scratch = (int64_t)lu;
    bitems[b][pos] = t;
    lu += 2ull * nb * nb;
  }
}

__global__ void k_gm_round_mid(TmxGState *G) {
  if (threadIdx.x != 0 || blockIdx.x != 0) {
    return;
  }
  for (int q = 0; q < TMX_GM_BUCKETS; ++q) {
    G->rng[q][1] = G->fill[q];
  }
  G->srng[1] = G->nslots;
}

// the next active list (act1) becomes the current one (act0)
__global__ void k_gm_swap(const TmxGState *__restrict__ G, const int32_t *__restrict__ next,
                          int32_t *cur, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n && p < G->cnt[2]) {
    cur[p] = next[p];
  }
}

__global__ void k_gm_end(TmxGState *G, cudaGraphConditionalHandle loop) {
  if (threadIdx.x != 0 || blockIdx.x != 0) {
    return;
  }
  G->cnt[0] = G->cnt[2];
  G->cnt[2] = 0;
  G->round_lo = G->round_hi;
  G->round_hi = G->cnt[1];
  G->k += 1;
  G->iter += 1;
  const bool active = G->cnt[0] > 0 && G->k <= G->last_order;
  const bool pending = G->round_hi > G->round_lo;
  // (a bound on the iterations: one per order, one more for the last round)
  const bool more = (active || pending) && G->iter <= G->max_iter;
  cudaGraphSetConditional(loop, more ? 1u : 0u);
}


// ------------------------------------------------------ launch wrappers --

void tmx_launch_gm_begin(TmxGState *G, TmxGIter *I, const int32_t *m0_sets, int min_order,
                         int glf, cudaStream_t stream) {
  k_gm_begin<<<1, 32, 0, stream>>>(G, I, m0_sets, min_order, glf);
}

void tmx_launch_gm_prep(const TmxGState *G, const TmxGIter *I, const int32_t *active, int n,
                        TmxSlot *slots, TmxItem *items, cudaStream_t stream) {
  k_gm_prep<<<(n + 127) / 128, 128, 0, stream>>>(G, I, active, n, slots, items);
}

void tmx_launch_gm_round(const TmxGmRoundArgs &a, cudaStream_t stream) {
  k_gm_round<<<(a.n + 127) / 128, 128, 0, stream>>>(
      a.G, a.done_list, a.done_ord, a.keep_tab, a.tpl_off, a.tpl, a.full_sets, a.tsize,
      a.glf, a.min_order, a.rslots, a.n, a.bitems, a.bcap, a.t_off, a.t_cap, a.lu_cap);
}

void tmx_launch_gm_round_mid(TmxGState *G, cudaStream_t stream) {
  k_gm_round_mid<<<1, 32, 0, stream>>>(G);
}

void tmx_launch_gm_swap(const TmxGState *G, const int32_t *next, int32_t *cur, int n,
                        cudaStream_t stream) {
  k_gm_swap<<<(n + 127) / 128, 128, 0, stream>>>(G, next, cur, n);
}

void tmx_launch_gm_end(TmxGState *G, cudaGraphConditionalHandle loop, cudaStream_t stream) {
  k_gm_end<<<1, 32, 0, stream>>>(G, loop);
}
