// Host-side launch wrappers of the CUDA kernels (internal).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tmx_internal.h"

// One Wigner d table set: all m in [m_lo, m_hi] at the lower-half nodes of
// the 2 ngauss Gauss-Legendre rule, n = 1..nmax.
struct TmxWigJob {
  int32_t nmax;
  int32_t ngauss;
  int32_t m_lo;
  int32_t m_hi;
  int64_t out; // offset (doubles) into the Wigner buffer
};

// Per-grain convergence state of the order loop (ConvergedSizeResources and
// the Q sums kept in TMatrixResource).
struct TmxChainState {
  double qsca, qext;   // m = 0 sums of the latest order
  double dqs_t, dqe_t; // TMatrixResource::_dQscattering/_dQextinction
  double dqs, dqe;     // ConvergedSizeResources::_dQs/_dQe
  int32_t nmax, ngauss;
  int32_t converged;
  int32_t status;
};

// node scalars and Bessel tables of every slot; ngmax >= every slot's
// ngauss, nmax_max >= every slot's nmax
void tmx_launch_tables(const TmxSlot *slots, int nslots, const TmxGrain *grains,
                       const double *gl_x, const double *gl_w,
                       const int64_t *gl_off, double *tab, double *nsc,
                       int bessel_start, int ngmax, int nmax_max,
                       cudaStream_t stream);

// device-driven form: slots [0, min(nslots, *nact)), each with *ng_dev nodes
// and order <= nmax_max
void tmx_launch_tables_dev(const TmxSlot *slots, int nslots, const int32_t *nact,
                           const int32_t *ng_dev, const TmxGrain *grains,
                           const double *gl_x, const double *gl_w,
                           const int64_t *gl_off, double *tab, double *nsc,
                           int bessel_start, int nmax_max, cudaStream_t stream);

void tmx_launch_wigner(const TmxWigJob *jobs, int njobs, int max_work,
                       const double *gl_x, const int64_t *gl_off, double *out,
                       cudaStream_t stream);

// block kernel: assembly + LU + solve for a list of (slot, m, class) items
struct TmxBlockArgs {
  const TmxItem *items;
  int nitems;
  const TmxSlot *slots;
  const TmxGrain *grains;
  const double *tab;
  const double *nsc;
  const double *wig;           // Wigner buffer
  const int64_t *wig_off;      // per Wigner set: offset of m = 0 (doubles)
  double2 *scratch;            // per-item Q / RgQ scratch
  double2 *tout;               // T-matrix storage (complex)
  double2 *diag;               // chain-mode diagonal buffer
  int32_t *status;             // per grain status bits
  int chunk_nodes;             // quadrature nodes per shared-memory chunk
  int max_nb;                  // largest class size in this launch
  double2 *lu = nullptr;       // if set: LU factors + pivots saved per item
                               // at the item's scratch offset (2 nb^2)
  int family = -1;             // tmx_block_family to run, -1: by max_nb
  // device-driven launches (CUDA graph): items [range[0], range[1]) of
  // `items` (clamped to nitems) instead of [0, nitems); at most max_ctas
  // CTAs (0: one item per warp or CTA)
  const int32_t *range = nullptr;
  int max_ctas = 0;
};
// largest class size each tmx_block_family can run
int tmx_block_family_capacity(int family);
size_t tmx_block_smem_bytes(int max_nb, int chunk_nodes);
void tmx_launch_blocks(const TmxBlockArgs &a, cudaStream_t stream);

// slots and m = 0 items of one order step from the active list
// buffer offsets of one order's slots in a (possibly speculative) group of
// orders: slot index, table/scalar/diagonal/scratch bases and strides
struct TmxChainBase {
  int32_t slot;
  int64_t tab, tab_stride;
  int64_t nsc, nsc_stride;
  int64_t diag, diag_stride;
  int64_t scr, scr_stride;
};
// nact_dev (may be NULL): the list's length on the device; positions
// p >= *nact_dev - base of this launch (for nactive, an upper bound) get empty
// slots
void tmx_launch_chain_prep(const int32_t *active, int nactive,
                           const int32_t *nact_dev, int base, int order,
                           int ngauss, int wig_n, const TmxChainBase &b,
                           TmxSlot *slots, TmxItem *items, cudaStream_t stream);

// convergence step for the active slots of one order
// m = 0 sums and the convergence test of one order; grains that continue go
// to next_active, grains whose order is final are appended to done_list
// (with that order in done_ord); grains already final are skipped
// (done_pos: the grain's position in `active`)
void tmx_launch_converge(const int32_t *active, int nactive,
                         const TmxSlot *slots, const double2 *diag,
                         TmxChainState *state, double tolerance, int order,
                         int last_order, int32_t *next_active,
                         int32_t *next_count, int32_t *done_list,
                         int32_t *done_ord, int32_t *done_pos,
                         int32_t *done_count, const int32_t *nact_dev,
                         int base, cudaStream_t stream,
                         const int32_t *order_dev = nullptr);

// state of the device-driven order loop (tmx_graph.cu), in device memory
#define TMX_GM_BUCKETS 5
#define TMX_GM_RSLOTS 8
struct TmxGState {
  unsigned long long t_used, lu_used; // T-matrix and LU storage handed out
  int32_t cnt[3];   // [0] list A length, [1] done-list length, [2] list B length
  int32_t loop_done;                  // a step found its input list empty
  int32_t next_k;                     // first order not yet evaluated
  int32_t snap_last;                  // done-list length after the latest step
  int32_t steps, rounds;              // order steps run, rounds fired
  int32_t kernels;                    // kernels the steps' and rounds' bodies ran
  int32_t cursor;                     // done entries handed to rounds so far
  // rounds run in round slots r = k mod TMX_GM_RSLOTS, several at once: the
  // done entries [rlo[r], rhi[r]) of slot r's round, its items per size
  // bucket and its round slots
  int32_t rlo[TMX_GM_RSLOTS], rhi[TMX_GM_RSLOTS];
  int32_t fill[TMX_GM_BUCKETS];       // items appended per size bucket
  int32_t rng[TMX_GM_RSLOTS][TMX_GM_BUCKETS][2];
  int32_t nslots, srng[TMX_GM_RSLOTS][2]; // round slots appended; each slot's
  int32_t overflow;                   // storage or arena ran out (bit mask)
};
// parameters of one order step, written by k_gm_begin
struct TmxGIter {
  int32_t order, ngauss, wig_n;
  int32_t m0_range[2]; // the m = 0 items of the active slots: [0, 4 active)
  TmxChainBase base;
};

// the device-driven loop's kernels (tmx_graph.cu)
struct TmxGmRoundArgs {
  TmxGState *G;
  int rs;                    // round slot (0 .. TMX_GM_RSLOTS - 1)
  const int32_t *done_list, *done_ord;
  const int64_t *keep_tab;
  const int32_t *tpl_off, *tpl, *full_sets;
  const int64_t *tsize;
  int glf, min_order;
  TmxSlot *rslots;
  int n;                     // grains of the batch (slot capacity)
  TmxItem *const *bitems;    // item array of each size bucket (device array)
  const int32_t *bcap;       // their capacities (device)
  int64_t *t_off;            // per grain: T-matrix offset
  unsigned long long t_cap, lu_cap;
};
// lists: `in` / `out` name the counts cnt[in] / cnt[out] of the step's input
// and output lists
void tmx_launch_gm_begin(TmxGState *G, TmxGIter *I, int k, int glf, int wig_n, int in, int out,
                         cudaStream_t stream);
void tmx_launch_gm_prep(const int32_t *nact, const TmxGIter *I, const int32_t *active, int n,
                        TmxSlot *slots, TmxItem *items, cudaStream_t stream);
void tmx_launch_gm_step_end(TmxGState *G, int32_t *snap, int32_t *outz, int j, int out,
                            int in, int next_k, int nk, cudaStream_t stream);
void tmx_launch_gm_relist(TmxGState *G, const int32_t *from, int32_t *to, int n, int in,
                          int out, cudaStream_t stream);
void tmx_launch_gm_round(const TmxGmRoundArgs &a, cudaStream_t stream);
void tmx_launch_gm_round_mid(TmxGState *G, int rs, cudaStream_t stream);
void tmx_launch_gm_tzero(const TmxGState *G, int rs, const TmxSlot *slots,
                         const int64_t *tsize, double2 *T, cudaStream_t stream);
void tmx_launch_gm_round_end(TmxGState *G, int nk, cudaStream_t stream);
// the chains' control kernels as graph kernel nodes (0 or -1)
int tmx_gm_add_cond(cudaGraph_t g, const cudaGraphNode_t *deps, size_t nd, cudaGraphNode_t *node,
                    TmxGState *G, int in, int k, cudaGraphConditionalHandle h1,
                    cudaGraphConditionalHandle h4, cudaGraphConditionalHandle h8, int has4,
                    int has8, int priority);
int tmx_gm_add_decide(cudaGraph_t g, const cudaGraphNode_t *deps, size_t nd,
                      cudaGraphNode_t *node, TmxGState *G, const int32_t *snap,
                      const int32_t *outz, int j, int last, int thr, int rmax, int rs,
                      cudaGraphConditionalHandle hform, cudaGraphConditionalHandle hexec,
                      int priority);

// copies of the final-order tables of the grains that became final in one
// group of orders, into the batch's table arena (k_keep_tables)
#define TMX_MAX_GROUP 8
struct TmxKeepArgs {
  const int32_t *done_list, *done_ord, *done_pos;
  const int32_t *counters;          // [1]: entries in the done list
  int32_t *next;                    // first entry not yet kept
  unsigned *ticket;                 // CTAs finished (last one resets it)
  int order0;                       // first order of the group
  TmxChainBase base[TMX_MAX_GROUP]; // table layout of each order of the group
  const double *tab, *nsc;          // the order loop's table buffers
  double *arena;
  long long cap;                    // arena capacity (doubles)
  unsigned long long *used;         // doubles reserved so far
  int64_t *keep_tab;                // per grain: arena offset (-1: none)
  int64_t *keep_q;                  // per done-list entry: the same
  // device-driven loop: the order and table layout of the (one-order) group
  // read on the device instead of order0 / base[0]
  const int32_t *order0_dev = nullptr;
  const TmxChainBase *base_dev = nullptr;
};
void tmx_launch_keep_tables(const TmxKeepArgs &K, int max_entries,
                            cudaStream_t stream);

// full Q sums over all m blocks (TMatrixQTask) of the grains of a block round: q_out[2 g], q_out[2 g + 1]
// for g = slots[s].grain
// (range: slots [range[0], range[1]) of the ns, read on the device; at most
// max_ctas CTAs, 0: one per slot)
void tmx_launch_qsums(const TmxSlot *slots, int ns, const double2 *T,
                      double *q_out, cudaStream_t stream,
                      const int32_t *range = nullptr, int max_ctas = 0);

// FP64 throughput probes (DFMA pipe and DMMA tensor pipe)
void tmx_launch_probe_dfma(double *out, int iters, int blocks,
                           cudaStream_t stream);
void tmx_launch_probe_dmma(double *out, int iters, int blocks,
                           cudaStream_t stream);

// host helpers shared by the drivers (tmx_host.cu)
void tmx_host_gauss_legendre(int order, double *points, double *weights);
int tmx_host_class_size(int N, int m, int cls);
int tmx_host_chunk_nodes(int max_nb);

// ------------------------------------------------------------ observables --

// per-grain descriptor of the observable kernels
struct TmxObsGrain {
  int32_t nmax;
  int32_t coef_set; // orientation coefficient set, -1: no averaging
  int64_t t_off;    // complex offset of the grain's T-matrix
  double k;         // wavenumber
  double r_ev;      // equal-volume radius
};

// cos, sin, 1/sin of a zenith angle as the reference's grids compute them
struct TmxAngle {
  double c, s, si;
};

// forward-amplitude job: S(theta_in -> theta_out) for nphi azimuths
struct TmxSJob {
  int32_t grain;
  int32_t angle_in;
  int32_t angle_out;
  int32_t nphi;
  int64_t phi0; // first e^{i phi} of the job in the azimuth table
  int64_t out;  // first S (4 complex each) of the job
};

// consecutive amplitude jobs of one grain handled by one CTA (at most 32)
struct TmxAmpGroup {
  int32_t grain;
  int32_t njobs;
  int64_t job0;
};

// Q job for one (grain, theta): main amplitude and, with the scattering
// subtraction, nacc x nacc amplitudes starting at s_acc
struct TmxQJob {
  int32_t grain;
  int32_t pad;
  int64_t out;
  int64_t s_main;
  int64_t s_acc;
};

void tmx_launch_cg(int nmax, const int64_t *cg_off, double *cg, double *work,
                   int blocks, cudaStream_t stream);
// source and destination arrays of up to four matrix sets processed by one
// launch (a T-matrix set and its tangents)
struct TmxMatSet {
  const double2 *src[4];
  double2 *dst[4];
};
// orientation average (coef_set >= 0) or copy of every grain's T-matrix,
// with the amplitude factors c_{n' n} folded in when fold != 0;
// work items (pair (n1, n2), grain) pair-major: pair q = (n1 - 1) pmax +
// n2 - 1 owns items [pstart[q], pstart[q + 1]), for the grains
// order[0 .. pstart[q + 1] - pstart[q]) (grains by descending nmax, so the
// grains of order >= max(n1, n2) come first); npairs = sum of nmax^2;
// mmax >= every nmax; nmat (1 or 4) sets src[k] -> dst[k]
void tmx_launch_orient_pairs(const TmxObsGrain *og, const int64_t *pstart,
                             const int32_t *order, int pmax, int64_t npairs,
                             const TmxMatSet &mats,
                             int nmat, const double *coeffs, int ncoef,
                             const int64_t *cg_off, const double *cg,
                             int cg_nmax, int mmax, int fold,
                             cudaStream_t stream);
// CTAs of the amplitude kernel at full occupancy for nbmax and nmat (its
// work slots: grid x nmat x 32 x (nbmax + 1) x 4 complex)
int tmx_amp_grid(int nbmax, int nmat);
// amplitudes of nmat (1 or 4) averaged sets: src[k] -> S at dst[k]
// wpi / wtau (may be NULL: the kernel runs the recurrences itself): the
// plan's pi and tau columns from tmx_launch_wigner_cols for nmax wnmax
void tmx_launch_amp(const TmxAmpGroup *groups, int ngroups, const TmxSJob *jobs,
                    const TmxObsGrain *og, const TmxMatSet &mats, int nmat,
                    const TmxAngle *angles, const double2 *phis, double2 *xslot,
                    int nbmax, int grid, const double *wpi, const double *wtau,
                    int wnmax, cudaStream_t stream);
// pi and tau columns of every (angle, m <= nmax): column (a, m) holds orders
// max(m, 1) .. nmax at ((a (nmax + 1) + m) nmax)
void tmx_launch_wigner_cols(const TmxAngle *angles, int nangles, int nmax,
                            double *pi, double *tau, cudaStream_t stream);
void tmx_launch_q_epilogue(const TmxQJob *jobs, int njobs, const TmxObsGrain *og,
                           const double2 *S, const double *wts, int nacc,
                           double *qout, int qstride, int do_abs, int do_ext,
                           cudaStream_t stream);
void tmx_launch_z_epilogue(int n, const double2 *S, double *zout,
                           cudaStream_t stream);
void tmx_launch_dq_epilogue(const TmxQJob *jobs, int njobs,
                            const TmxObsGrain *og, const double2 *S,
                            const double2 *dSm, const double2 *dSr,
                            const double2 *dSd, double *dq, cudaStream_t stream);
void tmx_launch_shape_avg(int ncells, int nshape, int nper, const double *in,
                          const double *w, double *out, cudaStream_t stream);

// ---------------------------------------------------------------- tangents --

// d/dp of every class block for p = refractive index (complex derivative),
// equal-volume radius, axis ratio: dT = -(dRgQ + T dQ) Q^-1 with the LU
// factors saved by the forward block kernel.
struct TmxTangentArgs {
  const TmxItem *items;
  int nitems;
  int nparams;                 // parameters per item (param = blockIdx.y)
  const TmxSlot *slots;
  const TmxGrain *grains;
  const double *tab;
  const double *nsc;
  const double *wig;
  const int64_t *wig_off;
  const double2 *lu;           // saved LU factors / pivots (forward)
  const double2 *T;            // forward T-matrices
  double2 *scratch;            // per (item, param): dQ, dRgQ (2 nb^2)
  int64_t scratch_stride;      // complex elements per parameter
  double2 *dT;                 // tangent T-matrices, one set per parameter
  int64_t dT_stride;           // complex elements per parameter set
  int chunk_nodes;
  int max_nb;
};
size_t tmx_tangent_smem_bytes(int max_nb, int chunk_nodes);
void tmx_launch_tangents(const TmxTangentArgs &a, cudaStream_t stream);
