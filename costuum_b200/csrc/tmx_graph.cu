// Device-driven batch (TMX_BATCH_GRAPH): the order loop and the block rounds
// of tmx_batch_compute as one CUDA graph, launched once; the host uploads the
// batch's descriptors, launches the graph and reads the results.
//
// Reference semantics are those of the host-driven loop (TaskManager.hpp:
// 1146-1197 chain of TMatrixM0Task per order, :1313-1327 TMatrixMAllTask
// once the order is final): every order step of every active grain, the
// convergence test in the reference's order, and the blocks of every m at
// the final order.
//
// The graph has two chains of conditional (IF) nodes, one node of each per
// order k = min_order .. maximum_order - 1:
//   loop chain (high priority)
//     k_gm_cond       which form of step k runs, if any (a grain is still
//                     active and k is not inside an earlier group of orders):
//                     one order, or with few grains left 4 or 8 orders at
//                     once as the host-driven loop speculates
//     IF step k:      k_gm_begin (step parameters, next list emptied),
//                     k_gm_prep (slots and m = 0 items of the active list),
//                     k_tables_dev, the m = 0 block launch, k_converge,
//                     k_keep_tables, k_gm_step_end (snapshot of the done list)
//   round chain (low priority), after step k, the previous round's formation
//   and the round TMX_GM_RSLOTS orders earlier (rounds run in round slots
//   k mod TMX_GM_RSLOTS, several at once)
//     k_gm_decide     whether to run a round now: at least a threshold of
//                     grains final and not yet in a round, or the loop over
//     IF form k:      k_gm_round (slots and items of those grains, every m
//                     and class, into per-size-bucket item arrays; T-matrix
//                     and LU offsets), k_gm_round_mid, k_gm_tzero (their
//                     T-matrices cleared)
//     IF run k:       one block launch per size bucket side by side,
//                     k_qsums, k_gm_round_end
// Nothing in the loop chain waits for a round, so rounds run beside the
// later orders, as the host-driven loop's rounds do on their streams; the
// lists alternate between two buffers by the parity of k - min_order.
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

// which form of order step k runs, if any: none while k is inside a group
// of orders an earlier step evaluated (k < next_k) or once the input list
// (count cnt[in]) is empty; else a group of 8 orders for at most 32 active
// grains, of 4 orders for at most 128 (where the graph has those forms: the
// group fits below the last order), one order otherwise -- the host-driven
// loop's speculation rule
__global__ void k_gm_cond(TmxGState *G, int in, int k, cudaGraphConditionalHandle h1,
                          cudaGraphConditionalHandle h4, cudaGraphConditionalHandle h8,
                          int has4, int has8) {
  if (threadIdx.x != 0 || blockIdx.x != 0) {
    return;
  }
  int form = 0;
  if (k >= G->next_k && !G->loop_done) {
    const int a = G->cnt[in];
    if (a <= 0) {
      G->loop_done = 1;
    } else {
      form = (has8 && a <= 32) ? 8 : (has4 && a <= 128) ? 4 : 1;
    }
  }
  // (a form the graph does not have has no IF node and no handle)
  cudaGraphSetConditional(h1, form == 1 ? 1u : 0u);
  if (has4) {
    cudaGraphSetConditional(h4, form == 4 ? 1u : 0u);
  }
  if (has8) {
    cudaGraphSetConditional(h8, form == 8 ? 1u : 0u);
  }
}

// end of a group of orders: the grains still active after its last order
// (list `out`) become the input list of the next step (list `in`, the same
// parity: the group's length is even)
__global__ void k_gm_relist(TmxGState *G, const int32_t *__restrict__ from, int32_t *to,
                            int n, int in, int out) {
  const int c = G->cnt[out];
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < min(c, n);
       p += gridDim.x * blockDim.x) {
    to[p] = from[p];
  }
}

// parameters of step k; the step's output list starts empty
__global__ void k_gm_begin(TmxGState *G, TmxGIter *I, int k, int glf, int wig_n, int in,
                           int out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) {
    return;
  }
  TmxGIter it;
  it.order = k;
  it.ngauss = glf * k;
  it.wig_n = wig_n;
  const int cm = (k + 1) / 2;
  it.m0_range[0] = 0;
  it.m0_range[1] = 4 * G->cnt[in];
  TmxChainBase &b = it.base;
  b.slot = 0;
  b.tab = b.nsc = b.diag = b.scr = 0;
  b.tab_stride = (int64_t)glf * k * k * TMX_NQ;
  b.nsc_stride = (int64_t)glf * k * TMX_NS;
  b.diag_stride = 2 * (int64_t)k;
  b.scr_stride = 2 * (int64_t)cm * cm;
  *I = it;
  G->cnt[out] = 0;
}

// slots and m = 0 items of every active position p < n (positions at or past
// the list's length *nact get an empty slot: order 0, no classes, no nodes)
__global__ void k_gm_prep(const int32_t *__restrict__ nact, const TmxGIter *__restrict__ I,
                          const int32_t *__restrict__ active, int n, TmxSlot *slots,
                          TmxItem *items) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) {
    return;
  }
  const TmxGIter it = *I;
  const bool valid = p < *nact;
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

// end of step j = k - min_order: the done list's length now (every entry
// and its kept tables complete), and whether the output list is empty
__global__ void k_gm_step_end(TmxGState *G, int32_t *snap, int32_t *outz, int j, int out,
                              int in, int next_k, int nk) {
  if (threadIdx.x != 0 || blockIdx.x != 0) {
    return;
  }
  snap[j] = G->cnt[1];
  outz[j] = (G->cnt[out] == 0) ? 1 : 0;
  if (in >= 0) {
    // (a group: its surviving list was copied into list `in`)
    G->cnt[in] = G->cnt[out];
  }
  G->snap_last = G->cnt[1];
  G->next_k = next_k;
  G->steps += 1;
  atomicAdd(&G->kernels, nk); // the kernels of this step's body (round
                              // bodies running beside it add theirs too)
}

// whether round j runs: the done entries that step j completed (or, if step
// j did not run, every entry) not yet in a round, at least `thr` of them
// while the loop continues (at most rmax per round), all of them once the
// loop is over (step j found its output list empty, did not run, or was the
// last order)
__global__ void k_gm_decide(TmxGState *G, const int32_t *__restrict__ snap,
                            const int32_t *__restrict__ outz, int j, int last, int thr,
                            int rmax, int rs, cudaGraphConditionalHandle hform,
                            cudaGraphConditionalHandle hexec) {
  if (threadIdx.x != 0 || blockIdx.x != 0) {
    return;
  }
  const bool ran = snap[j] >= 0;
  const int avail = ran ? snap[j] : G->snap_last;
  const bool ended = !ran || outz[j] != 0 || last != 0;
  const int pending = avail - G->cursor;
  const bool fire = pending > 0 && (ended || pending >= thr);
  if (fire) {
    G->rlo[rs] = G->cursor;
    G->rhi[rs] = ended ? avail : min(avail, G->cursor + rmax);
    G->cursor = G->rhi[rs];
    for (int q = 0; q < TMX_GM_BUCKETS; ++q) {
      G->rng[rs][q][0] = G->fill[q];
      G->rng[rs][q][1] = G->fill[q];
    }
    G->srng[rs][0] = G->nslots;
    G->srng[rs][1] = G->nslots;
    G->rounds += 1;
  }
  cudaGraphSetConditional(hform, fire ? 1u : 0u);
  cudaGraphSetConditional(hexec, fire ? 1u : 0u);
}

// The round: one thread per done entry of [round_lo, round_hi). A grain's
// items come from the template of its order (tpl_off[N] .. tpl_off[N + 1]
// in tpl, (m << 8 | class) and the class size), into the item array of
// their size bucket; its T-matrix and each item's LU factors get offsets
// from bump counters. A grain without kept tables or beyond the T / LU
// capacity sets the overflow flag (the host then recomputes the batch).
__global__ void k_gm_round(TmxGState *G, int rs, const int32_t *__restrict__ done_list,
                           const int32_t *__restrict__ done_ord,
                           const int64_t *__restrict__ keep_tab,
                           const int32_t *__restrict__ tpl_off,
                           const int32_t *__restrict__ tpl,
                           const int32_t *__restrict__ full_sets,
                           const int64_t *__restrict__ tsize, int glf, int min_order,
                           TmxSlot *rslots, int nslot_cap, TmxItem *const *bitems,
                           const int32_t *__restrict__ bcap, int64_t *t_off,
                           unsigned long long t_cap, unsigned long long lu_cap) {
  const int q = G->rlo[rs] + blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G->rhi[rs]) {
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

__global__ void k_gm_round_mid(TmxGState *G, int rs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) {
    return;
  }
  for (int q = 0; q < TMX_GM_BUCKETS; ++q) {
    G->rng[rs][q][1] = G->fill[q];
  }
  G->srng[rs][1] = G->nslots;
}

// The T-matrix ranges of the round's slots [srng[0], srng[1]) start at
// zero: the parity classes write only their own entries of a block, the
// others are zero by symmetry (the host-driven rounds clear their range the
// same way). One CTA per slot at a time, 16-byte stores.
__global__ void k_gm_tzero(const TmxGState *__restrict__ G, int rs,
                           const TmxSlot *__restrict__ slots,
                           const int64_t *__restrict__ tsize, double2 *T) {
  const int lo = G->srng[rs][0], hi = G->srng[rs][1];
  for (int s = lo + blockIdx.x; s < hi; s += gridDim.x) {
    const TmxSlot sl = slots[s];
    if (sl.nmax <= 0) {
      continue;
    }
    double2 *t = T + sl.tout;
    const int64_t ts = tsize[sl.nmax];
    for (int64_t u = threadIdx.x; u < ts; u += blockDim.x) {
      t[u] = make_double2(0., 0.);
    }
  }
}

// the round's done entries are consumed
__global__ void k_gm_round_end(TmxGState *G, int nk) {
  if (threadIdx.x != 0 || blockIdx.x != 0) {
    return;
  }
  atomicAdd(&G->kernels, nk); // the kernels of this round's bodies
}


// ------------------------------------------------------ launch wrappers --

void tmx_launch_gm_begin(TmxGState *G, TmxGIter *I, int k, int glf, int wig_n, int in, int out,
                         cudaStream_t stream) {
  k_gm_begin<<<1, 32, 0, stream>>>(G, I, k, glf, wig_n, in, out);
}

void tmx_launch_gm_prep(const int32_t *nact, const TmxGIter *I, const int32_t *active, int n,
                        TmxSlot *slots, TmxItem *items, cudaStream_t stream) {
  k_gm_prep<<<(n + 127) / 128, 128, 0, stream>>>(nact, I, active, n, slots, items);
}

void tmx_launch_gm_step_end(TmxGState *G, int32_t *snap, int32_t *outz, int j, int out,
                            int in, int next_k, int nk, cudaStream_t stream) {
  k_gm_step_end<<<1, 32, 0, stream>>>(G, snap, outz, j, out, in, next_k, nk);
}

void tmx_launch_gm_relist(TmxGState *G, const int32_t *from, int32_t *to, int n, int in,
                          int out, cudaStream_t stream) {
  k_gm_relist<<<std::max(1, std::min((n + 255) / 256, 148)), 256, 0, stream>>>(G, from, to,
                                                                             n, in, out);
}

void tmx_launch_gm_round(const TmxGmRoundArgs &a, cudaStream_t stream) {
  k_gm_round<<<(a.n + 127) / 128, 128, 0, stream>>>(
      a.G, a.rs, a.done_list, a.done_ord, a.keep_tab, a.tpl_off, a.tpl, a.full_sets, a.tsize,
      a.glf, a.min_order, a.rslots, a.n, a.bitems, a.bcap, a.t_off, a.t_cap, a.lu_cap);
}

void tmx_launch_gm_round_mid(TmxGState *G, int rs, cudaStream_t stream) {
  k_gm_round_mid<<<1, 32, 0, stream>>>(G, rs);
}

void tmx_launch_gm_tzero(const TmxGState *G, int rs, const TmxSlot *slots,
                         const int64_t *tsize, double2 *T, cudaStream_t stream) {
  k_gm_tzero<<<148 * 4, 256, 0, stream>>>(G, rs, slots, tsize, T);
}

void tmx_launch_gm_round_end(TmxGState *G, int nk, cudaStream_t stream) {
  k_gm_round_end<<<1, 32, 0, stream>>>(G, nk);
}

// The two control kernels of the top-level chains as graph kernel nodes
// (they set the condition of the IF node that follows them), with the
// given dependencies and execution priority.
static int add_kernel_node(cudaGraph_t g, const cudaGraphNode_t *deps, size_t nd,
                           cudaGraphNode_t *node, void *func, void **args, int priority) {
  cudaKernelNodeParams p = {};
  p.func = func;
  p.gridDim = dim3(1);
  p.blockDim = dim3(32);
  p.sharedMemBytes = 0;
  p.kernelParams = args;
  p.extra = nullptr;
  if (cudaGraphAddKernelNode(node, g, deps, nd, &p) != cudaSuccess) {
    return -1;
  }
  cudaKernelNodeAttrValue v = {};
  v.priority = priority;
  if (cudaGraphKernelNodeSetAttribute(*node, cudaKernelNodeAttributePriority, &v) !=
      cudaSuccess) {
    return -1;
  }
  return 0;
}

int tmx_gm_add_cond(cudaGraph_t g, const cudaGraphNode_t *deps, size_t nd, cudaGraphNode_t *node,
                    TmxGState *G, int in, int k, cudaGraphConditionalHandle h1,
                    cudaGraphConditionalHandle h4, cudaGraphConditionalHandle h8, int has4,
                    int has8, int priority) {
  void *args[] = {&G, &in, &k, &h1, &h4, &h8, &has4, &has8};
  return add_kernel_node(g, deps, nd, node, (void *)k_gm_cond, args, priority);
}

int tmx_gm_add_decide(cudaGraph_t g, const cudaGraphNode_t *deps, size_t nd,
                      cudaGraphNode_t *node, TmxGState *G, const int32_t *snap,
                      const int32_t *outz, int j, int last, int thr, int rmax, int rs,
                      cudaGraphConditionalHandle hform, cudaGraphConditionalHandle hexec,
                      int priority) {
  void *args[] = {&G, &snap, &outz, &j, &last, &thr, &rmax, &rs, &hform, &hexec};
  return add_kernel_node(g, deps, nd, node, (void *)k_gm_decide, args, priority);
}
