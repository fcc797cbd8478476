// Block kernel: for one (grain, m, parity class) work item, assemble the
// class sub-matrices of Q and RgQ by quadrature, factor Q with partial
// pivoting in shared memory and solve T_c Q_c = -RgQ_c.
//
// Reference semantics (CosTuuM):
//   assembly  TMatrixM0Task::execute   src/TMatrixResource.hpp:601-709 (m=0)
//             TMatrixMAllTask::execute src/TMatrixResource.hpp:934-1100
//   inversion Matrix::plu_inverse      src/Matrix.hpp:261-384
//   T         T = -RgQ Q^-1            src/TMatrixResource.hpp:712-730
//
// Restructuring (same mathematics):
//  * Parity classes. Q_m has non-zero entries only where the row label
//    (i + n) % 2 equals the column label (m >= 1), and is block diagonal in i
//    for m = 0. Partial pivoting never picks a row of another class (those
//    entries are exact zeros) and elimination never mixes classes, so the
//    reference's LU of the full 2nb x 2nb block performs, entry for entry,
//    the LUs of the independent classes. Each class is one work item here.
//  * Assembly as a GEMM. Every entry is sum_g sum_{t<4} F_t(g, n1) W_t(g, n2)
//    with A-side vectors built from h_n1 = j + i y (or j alone for RgQ) and
//    B-side vectors built from j_n2(m k r); see build_chunk().
//  * T = -RgQ Q^-1 by two triangular solves on the LU factors instead of the
//    explicit inverse followed by a product.
#include <algorithm>

#include "tmx_blocks_common.cuh"


// Build the A-side (F) and B-side (W) vectors of nodes [g0, g0 + G).
//   F1 = a d h, F2 = a dd h, F3 = a d dh, F4 = a (dd dh + n(n+1) drr/kr d h)
//   G1 = a d dj~, G2 = a (dd dj~ + drr/(m k r) n(n+1) d j~), G3 = a d j~,
//   G4 = a dd j~  (j~ = j_n(m k r), dj~ its derivative form)
//   alpha = w r^2, mu = m^2 / sin^2, beta = m w r^2 / sin
//   Q11: W = (k2mr a mu G1, k2mr a G2, -k2 a mu G3, -k2 a G4)
//   Q22: W = (k2 a mu G1, k2 a G2, -k2mr a mu G3, -k2mr a G4)
//   Q12: W = i (k2mr b G4, k2mr b G3, k2 b G2, k2 b G1)
//   Q21: W = i (k2 b G4, k2 b G3, k2mr b G2, k2mr b G1)
// This is the expansion of the J11, J12, J21, J22 terms of
// TMatrixResource.hpp:993-1097 into products of one n1 factor and one n2
// factor per node.
// A-side vectors (F^j, F^y) of row member a at node g, stored to f[t * ts].
// LEAN: without the factor a_n (the caller scales the finished entries by
// a_n1 a_n2) and, for m = 0, only the terms 1 and 3 that survive mu = 0.
template <bool LEAN = false>
__device__ __forceinline__ void a_side_row(double j, double dj, double y,
                                           double dy, double d, double dd,
                                           const double *s, int n, cplx *f,
                                           int ts, int m) {
  const double nn = n * (n + 1.);
  const double q = nn * s[TMX_NS_DRR] * s[TMX_NS_KRINV] * d;
  if (LEAN) {
    if (m != 0) {
      f[0] = mkc(d * j, d * y);
      f[2 * ts] = mkc(d * dj, d * dy);
    }
    f[ts] = mkc(dd * j, dd * y);
    f[3 * ts] = mkc(dd * dj + q * j, dd * dy + q * y);
    return;
  }
  const double an = a_n(n);
  f[0] = mkc(an * d * j, an * d * y);
  f[ts] = mkc(an * dd * j, an * dd * y);
  f[2 * ts] = mkc(an * d * dj, an * d * dy);
  f[3 * ts] = mkc(an * (dd * dj + q * j), an * (dd * dy + q * y));
}

template <bool LEAN = false>
__device__ __forceinline__ void a_side(const ClassDesc &D, int a, int N, int g,
                                       const double *__restrict__ T,
                                       const double *__restrict__ S,
                                       const double *__restrict__ Wg, cplx *f,
                                       int ts, int m = 1) {
  int i, n;
  member(D, a, i, n);
  const double *t = T + ((int64_t)g * N + (n - 1)) * TMX_NQ;
  const double *w = Wg + ((int64_t)g * N + (n - 1)) * 2;
  a_side_row<LEAN>(t[TMX_Q_J], t[TMX_Q_DJ], t[TMX_Q_Y], t[TMX_Q_DY], w[0], w[1],
                   S + (int64_t)g * TMX_NS, n, f, ts, m);
}

// B-side vectors of column member b at node g for each row group, stored to
// w[rg * gs + t * ts] (rg = 0 rows of block index D.iA, rg = 1 rows of D.iB).
// LEAN as for a_side.
template <bool LEAN = false>
__device__ __forceinline__ void b_side_row(const ClassDesc &D, int ib, int n,
                                           int m, cplx jm, cplx djm, double d,
                                           double dd, const double *s,
                                           int ngroups, double k2, cplx k2mr,
                                           cplx *w, int ts, int gs) {
  const double an = LEAN ? 1. : a_n(n);
  const double nn = n * (n + 1.);
  const cplx kmi = mkc(s[TMX_NS_KRMRINV_RE], s[TMX_NS_KRMRINV_IM]);
  const cplx G1 = cscale(djm, an * d);
  const cplx G2 = cscale(
      cadd(cscale(djm, dd), cscale(cmul(kmi, jm), s[TMX_NS_DRR] * nn * d)), an);
  const cplx G3 = cscale(jm, an * d);
  const cplx G4 = cscale(jm, an * dd);
  const double wr2 = s[TMX_NS_W] * s[TMX_NS_R2];
  const double mu = (double)(m * m) * s[TMX_NS_SIN2INV];
  const double beta = s[TMX_NS_SININV] * m * wr2;
  for (int rg = 0; rg < ngroups; ++rg) {
    const int ia = (rg == 0) ? D.iA : D.iB;
    cplx *wr = w + rg * gs;
    if (ia == ib) {
      // diagonal-type block: Q11 (i = 0) or Q22 (i = 1)
      const cplx chi = (ia == 0) ? k2mr : mkc(k2, 0.);
      const cplx clo = (ia == 0) ? mkc(-k2, 0.) : mkc(-k2mr.x, -k2mr.y);
      if (!LEAN || m != 0) {
        wr[0] = cmul(chi, cscale(G1, wr2 * mu));
        wr[2 * ts] = cmul(clo, cscale(G3, wr2 * mu));
      }
      wr[ts] = cmul(chi, cscale(G2, wr2));
      wr[3 * ts] = cmul(clo, cscale(G4, wr2));
    } else {
      // off-diagonal block: Q12 (ia = 0, ib = 1) or Q21 (ia = 1, ib = 0)
      const cplx c1 = (ia == 0) ? k2mr : mkc(k2, 0.);
      const cplx c2 = (ia == 0) ? mkc(k2, 0.) : k2mr;
      const cplx ic1 = mkc(-c1.y * beta, c1.x * beta); // i c1 beta
      const cplx ic2 = mkc(-c2.y * beta, c2.x * beta);
      wr[0] = cmul(ic1, G4);
      wr[ts] = cmul(ic1, G3);
      wr[2 * ts] = cmul(ic2, G2);
      wr[3 * ts] = cmul(ic2, G1);
    }
  }
}

template <bool LEAN = false>
__device__ __forceinline__ void b_side(const ClassDesc &D, int b, int N, int m,
                                       int g, int ngroups,
                                       const double *__restrict__ T,
                                       const double *__restrict__ S,
                                       const double *__restrict__ Wg, double k2,
                                       cplx k2mr, cplx *w, int ts, int gs) {
  int ib, n;
  member(D, b, ib, n);
  const double *t = T + ((int64_t)g * N + (n - 1)) * TMX_NQ;
  const double *wg = Wg + ((int64_t)g * N + (n - 1)) * 2;
  b_side_row<LEAN>(D, ib, n, m, mkc(t[TMX_Q_JM_RE], t[TMX_Q_JM_IM]),
                   mkc(t[TMX_Q_DJM_RE], t[TMX_Q_DJM_IM]), wg[0], wg[1],
                   S + (int64_t)g * TMX_NS, ngroups, k2, k2mr, w, ts, gs);
}

// zero A-side / B-side entries (padding and nodes past ngauss)
__device__ __forceinline__ void zero_side(cplx *f, int ts, int nt) {
  for (int t = 0; t < nt; ++t) {
    f[t * ts] = mkc(0., 0.);
  }
}

template <int TC>
__device__ void build_chunk(const ClassDesc &D, const AsmLayout &L, int N,
                            int m, int ng, int g0, const double *__restrict__ T,
                            const double *__restrict__ S,
                            const double *__restrict__ Wg, double k2,
                            cplx k2mr, cplx *Fs, cplx *Ws) {
  const int G = L.G;
  // A side
  for (int u = threadIdx.x; u < G * L.NRp; u += blockDim.x) {
    const int gl = u / L.NRp;
    const int pr = u % L.NRp;
    const int g = g0 + gl;
    const int a = padded_member(D, pr);
    cplx *fp = Fs + (int64_t)(4 * gl) * L.NRp + pr;
    if (a >= 0 && g < ng) {
      a_side(D, a, N, g, T, S, Wg, fp, L.NRp);
    } else {
      zero_side(fp, L.NRp, 4);
    }
  }
  // B side
  const int ncolp = L.CT * TC;
  for (int u = threadIdx.x; u < G * ncolp; u += blockDim.x) {
    const int gl = u / ncolp;
    const int b = u % ncolp;
    const int g = g0 + gl;
    cplx *wp = Ws + (int64_t)(4 * gl) * ncolp + b;
    const int gs = 4 * G * ncolp;
    if (b < D.nb && g < ng) {
      b_side(D, b, N, m, g, L.ngroups, T, S, Wg, k2, k2mr, wp, ncolp, gs);
    } else {
      for (int rg = 0; rg < L.ngroups; ++rg) {
        zero_side(wp + rg * gs, ncolp, 4);
      }
    }
  }
}

extern __shared__ __align__(16) unsigned char tmx_smem[];

// one item `it` by the whole CTA (every thread calls it; the early returns
// are uniform over the CTA)
template <int TR, int TC, int NT>
__device__ __forceinline__ void block_item(const TmxBlockArgs &A, int it,
                                           size_t smem_bytes) {
  const TmxItem item = A.items[it];
  const TmxSlot sl = A.slots[item.slot];
  const TmxGrain G = A.grains[sl.grain];
  const int N = sl.nmax;
  const int ng = sl.ngauss;
  const int m = item.m;
  const ClassDesc D = describe<TR>(N, m, item.cls);
  const int nb = D.nb;
  if (nb <= 0) {
    return;
  }
  // (shared memory is sized for classes of at most max_nb members)
  if (nb > TMX_MAX_NB || nb > A.max_nb) {
    if (threadIdx.x == 0) {
      atomicOr(&A.status[sl.grain], TMX_ST_TOO_LARGE);
    }
    return;
  }
  const double *T = A.tab + sl.tab;
  const double *S = A.nsc + sl.nsc;
  const double *Wg = A.wig + A.wig_off[sl.wig_n] + (int64_t)m * ng * N * 2;
  const double k2 = G.k * G.k;
  const cplx k2mr = mkc(G.mr * k2, G.mi * k2);
  cplx *Qs = A.scratch + item.scratch;
  cplx *Rs = Qs + (int64_t)nb * nb;

  // ------------------------------------------------------------ assembly
  AsmLayout L;
  L.G = A.chunk_nodes;
  L.NRp = D.NRp;
  L.CT = (nb + TC - 1) / TC;
  L.ncol = L.CT * TC;
  L.ngroups = (D.R1 > 0 && m > 0) ? 2 : 1;
  const int RT = D.NRp / TR;
  cplx *Fs = reinterpret_cast<cplx *>(tmx_smem);
  cplx *Ws = Fs + (int64_t)4 * L.G * L.NRp;
  const int ntiles = RT * L.CT;
  const int tstep = (m == 0) ? 2 : 1; // m = 0: mu = 0 kills t = 0, 2
  const int t0 = (m == 0) ? 1 : 0;
  for (int tile0 = 0; tile0 < ntiles; tile0 += NT) {
    const int tile = tile0 + threadIdx.x;
    const bool active = tile < ntiles;
    const int ct = active ? tile % L.CT : 0;
    const int rt = active ? tile / L.CT : 0;
    const int rg = (rt * TR < D.R0p) ? 0 : 1;
    double aj[TR][TC][2], ay[TR][TC][2];
#pragma unroll
    for (int r = 0; r < TR; ++r) {
#pragma unroll
      for (int c = 0; c < TC; ++c) {
        aj[r][c][0] = aj[r][c][1] = ay[r][c][0] = ay[r][c][1] = 0.;
      }
    }
    for (int g0 = 0; g0 < ng; g0 += L.G) {
      __syncthreads();
      build_chunk<TC>(D, L, N, m, ng, g0, T, S, Wg, k2, k2mr, Fs, Ws);
      __syncthreads();
      if (active) {
        const int kmax = 4 * min(L.G, ng - g0);
        for (int kk = t0; kk < kmax; kk += tstep) {
          const cplx *fr = Fs + (int64_t)kk * L.NRp + rt * TR;
          const cplx *wr = Ws + ((int64_t)rg * 4 * L.G + kk) * L.ncol + ct;
          cplx f[TR], w[TC];
#pragma unroll
          for (int r = 0; r < TR; ++r) {
            f[r] = fr[r];
          }
#pragma unroll
          for (int c = 0; c < TC; ++c) {
            w[c] = wr[c * L.CT];
          }
#pragma unroll
          for (int r = 0; r < TR; ++r) {
#pragma unroll
            for (int c = 0; c < TC; ++c) {
              aj[r][c][0] = fma(f[r].x, w[c].x, aj[r][c][0]);
              aj[r][c][1] = fma(f[r].x, w[c].y, aj[r][c][1]);
              ay[r][c][0] = fma(f[r].y, w[c].x, ay[r][c][0]);
              ay[r][c][1] = fma(f[r].y, w[c].y, ay[r][c][1]);
            }
          }
        }
      }
    }
    if (active) {
#pragma unroll
      for (int r = 0; r < TR; ++r) {
        const int a = padded_member(D, rt * TR + r);
        if (a < 0) {
          continue;
        }
#pragma unroll
        for (int c = 0; c < TC; ++c) {
          const int b = ct + c * L.CT;
          if (b >= nb) {
            continue;
          }
          // Q = G^j + i G^y, RgQ = G^j
          Qs[(int64_t)a * nb + b] =
              mkc(aj[r][c][0] - ay[r][c][1], aj[r][c][1] + ay[r][c][0]);
          Rs[(int64_t)a * nb + b] = mkc(aj[r][c][0], aj[r][c][1]);
        }
      }
    }
  }
  __syncthreads();

  // ------------------------------------------------------------------ LU
  // The factors live in shared memory (odd stride: conflict-free column
  // access) when they fit beside a chunk of at least 8 right-hand-side rows;
  // larger classes factor Q_c in place in its global scratch and solve on
  // -RgQ_c in place (L2-resident), with only the pivots in shared memory.
  const int lda_s = nb | 1;
  size_t lu_need = ((size_t)nb * lda_s + nb) * sizeof(cplx) + (3 * nb + 1) * sizeof(int);
  lu_need = (lu_need + 15) & ~(size_t)15;
  const bool lu_global =
      lu_need + (size_t)(nb < 8 ? nb : 8) * lda_s * sizeof(cplx) > smem_bytes;
  const int lda = lu_global ? nb : lda_s;
  cplx *Am = lu_global ? Qs : reinterpret_cast<cplx *>(tmx_smem);
  cplx *uinv = lu_global ? reinterpret_cast<cplx *>(tmx_smem) : Am + (int64_t)nb * lda;
  int *piv = reinterpret_cast<int *>(uinv + nb);
  int *perm = piv + nb;
  int *flag = perm + nb;
  cplx *X = lu_global ? Rs : reinterpret_cast<cplx *>(tmx_smem + lu_need);
  int Rchunk = lu_global ? nb : (int)((smem_bytes - lu_need) / (sizeof(cplx) * lda));
  if (Rchunk > nb) {
    Rchunk = nb;
  }
  if (!lu_global) {
    for (int u = threadIdx.x; u < nb * nb; u += blockDim.x) {
      Am[(u / nb) * lda + (u % nb)] = Qs[u];
    }
  }
  if (threadIdx.x == 0) {
    *flag = 0;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  for (int i = 0; i < nb; ++i) {
    if (warp == 0) {
      double best = -1.;
      int bi = i;
      for (int j = i + lane; j < nb; j += 32) {
        const double v = cabs_dev(Am[j * lda + i]);
        if (v > best) {
          best = v;
          bi = j;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ov > best || (ov == best && oi < bi)) {
          best = ov;
          bi = oi;
        }
      }
      if (lane == 0) {
        piv[i] = bi;
        if (!(best > 0.)) {
          *flag = 1;
        }
      }
    }
    __syncthreads();
    const int ip = piv[i];
    if (ip != i) {
      for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const cplx t = Am[i * lda + j];
        Am[i * lda + j] = Am[ip * lda + j];
        Am[ip * lda + j] = t;
      }
      __syncthreads();
    }
    const cplx pinv = cinv_lu(Am[i * lda + i]);
    for (int j = i + 1 + threadIdx.x; j < nb; j += blockDim.x) {
      Am[j * lda + i] = cmul(Am[j * lda + i], pinv);
    }
    __syncthreads();
    const int rem = nb - i - 1;
    for (int u = threadIdx.x; u < rem * rem; u += blockDim.x) {
      const int j = i + 1 + u / rem;
      const int k = i + 1 + u % rem;
      Am[j * lda + k] = csub(Am[j * lda + k], cmul(Am[j * lda + i], Am[i * lda + k]));
    }
    __syncthreads();
  }
  for (int j = threadIdx.x; j < nb; j += blockDim.x) {
    uinv[j] = cinv_lu(Am[j * lda + j]);
  }
  if (threadIdx.x == 0) {
    // column exchanges of Matrix::plu_inverse step 4, as a gather index
    for (int j = 0; j < nb; ++j) {
      perm[j] = j;
    }
    for (int j = nb - 1; j >= 0; --j) {
      const int p = piv[j];
      const int t = perm[j];
      perm[j] = perm[p];
      perm[p] = t;
    }
    if (*flag) {
      atomicOr(&A.status[sl.grain], TMX_ST_SINGULAR);
    }
  }
  __syncthreads();
  if (A.lu) {
    // factors (unit-lower L below, U on and above the diagonal) and the
    // column gather index, for the tangent solves
    cplx *Ls = A.lu + item.scratch;
    for (int u = threadIdx.x; u < nb * nb; u += blockDim.x) {
      Ls[u] = Am[(u / nb) * lda + (u % nb)];
    }
    int *ps = reinterpret_cast<int *>(Ls + (int64_t)nb * nb);
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
      ps[j] = perm[j];
    }
  }

  // --------------------------------------------- solve T_c Q_c = -RgQ_c
  const bool chain = sl.tout < 0;
  for (int r0 = 0; r0 < nb; r0 += Rchunk) {
    const int R = min(Rchunk, nb - r0);
    // (in place when X is Rs itself: each element is read and written by
    // the same thread)
    for (int u = threadIdx.x; u < R * nb; u += blockDim.x) {
      const cplx v = Rs[(int64_t)(r0 + u / nb) * nb + (u % nb)];
      X[(u / nb) * lda + (u % nb)] = mkc(-v.x, -v.y);
    }
    __syncthreads();
    // Z U = X (forward over columns)
    for (int j = 0; j < nb; ++j) {
      for (int r = threadIdx.x; r < R; r += blockDim.x) {
        X[r * lda + j] = cmul(X[r * lda + j], uinv[j]);
      }
      __syncthreads();
      const int rem = nb - j - 1;
      for (int u = threadIdx.x; u < R * rem; u += blockDim.x) {
        const int r = u / rem;
        const int k = j + 1 + u % rem;
        X[r * lda + k] = csub(X[r * lda + k], cmul(X[r * lda + j], Am[j * lda + k]));
      }
      __syncthreads();
    }
    // Y L = Z (backward over columns, L unit lower)
    for (int j = nb - 1; j >= 1; --j) {
      for (int u = threadIdx.x; u < R * j; u += blockDim.x) {
        const int r = u / j;
        const int k = u % j;
        X[r * lda + k] = csub(X[r * lda + k], cmul(X[r * lda + j], Am[j * lda + k]));
      }
      __syncthreads();
    }
    // write out: T_c[a][b] = Y[a][perm[b]]
    if (chain) {
      for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const int a = r0 + r;
        int ia, na;
        member(D, a, ia, na);
        A.diag[sl.diag + ia * N + (na - 1)] = X[r * lda + perm[a]];
      }
    } else {
      cplx *Tb = A.tout + sl.tout + block_offset(N, m);
      const int w2 = 2 * D.nbb;
      for (int u = threadIdx.x; u < R * nb; u += blockDim.x) {
        const int r = u / nb;
        const int b = u % nb;
        const int a = r0 + r;
        int ia, na, ib, nbn;
        member(D, a, ia, na);
        member(D, b, ib, nbn);
        const int row = ia * D.nbb + (na - D.nmin);
        const int col = ib * D.nbb + (nbn - D.nmin);
        Tb[(int64_t)row * w2 + col] = X[r * lda + perm[b]];
      }
    }
    __syncthreads();
  }
}

template <int TR, int TC, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_blocks(TmxBlockArgs A, size_t smem_bytes) {
  const int ilo = A.range ? A.range[0] : 0;
  const int ihi = A.range ? min(A.range[1], A.nitems) : A.nitems;
  for (int it = ilo + blockIdx.x; it < ihi; it += gridDim.x) {
    block_item<TR, TC, NT>(A, it, smem_bytes);
    // shared memory is reused by the next item
    __syncthreads();
  }
}

// ------------------------------------------------- warp-per-item variant --
//
// Classes of at most 16 members (nearly every item of grains up to order 32)
// are too small for a CTA: one warp owns one item from assembly to write-out
// and synchronises with __syncwarp only, so four independent items share a
// CTA. Assembly: lane (rt, ct) = (lane / 4, lane % 4) accumulates rows
// rt * TR .. rt * TR + TR - 1 and columns ct, ct + 4, .. of the class matrix
// over warp-private chunks of WG nodes. LU: lane r updates row r; the pivot
// column's maximum is a shuffle reduction (first maximum wins, as
// in Matrix::plu_inverse) and the factors stay in warp-private shared
// memory. Solve: lane r owns row r of -RgQ_c and runs both triangular solves
// on it against the factors, so no lane waits on another.

#ifndef TMX_WG
#define TMX_WG 4 // quadrature nodes per warp chunk (a multiple of 4)
#endif
// resident CTAs of four warps per SM the warp kernels are compiled for
// (register budget 65536 / (128 x MINB) per thread)
#ifndef TMX_WARP_DFMA_MINB
#define TMX_WARP_DFMA_MINB 4
#endif
#ifndef TMX_WARP_DMMA_MINB
#define TMX_WARP_DMMA_MINB 3
#endif

template <int NBM>
__host__ __device__ constexpr int warp_elems() {
  // chunk buffers F[WG][4][NBM] + W[2][WG][4][NBM]; the LU phase reuses them
  // for Q, RgQ ([NBM][NBM + 1] each), 1/U_jj and the pivot/gather indices
  return 12 * TMX_WG * NBM;
}

// Staging area of the next chunk's table rows (complex units): per node and
// class member one row of TMX_ROW doubles (the Bessel row j, j', y, y', j~,
// j~' and the Wigner pair d, d'; 80 bytes, so 16-byte reads of consecutive
// members hit distinct banks), and the node's scalar row (TMX_NS doubles).
#define TMX_ROW 10
template <int NBM>
__host__ __device__ constexpr int warp_stage_elems() {
  return TMX_WG * (NBM * TMX_ROW + TMX_NS) / 2;
}

// 16-byte asynchronous global -> shared copies (L2 only)
__device__ __forceinline__ void cp16(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Copies of one item's table rows into the staging area. Each lane owns up
// to SL_MAX 16-byte pieces of the member rows (piece p < 4 of the Bessel row
// of member a, or p = 4: its Wigner pair) and one piece of the node scalars;
// their source addresses at node 0 and their per-node strides are set up
// once per item, so a chunk costs one add and one copy per piece and node.
// Rows start on 16-byte boundaries: table offsets are multiples of TMX_NQ
// (8) doubles, Wigner offsets of 2 and node-scalar offsets of TMX_NS (16).
template <int NBM>
struct StagePlan {
  static constexpr int SL_MAX = (NBM * 5 + 31) / 32;
  // TMX_WG nodes x TMX_NS / 2 pieces of node scalars, SS per lane
  static constexpr int SS = TMX_WG * (TMX_NS / 2) / 32;
  static_assert(SS * 32 == TMX_WG * (TMX_NS / 2), "node-scalar pieces per lane");
  const double *src[SL_MAX]; // piece at node 0
  int stride[SL_MAX];        // doubles per node
  int dst[SL_MAX];           // double offset in the stage (node 0); -1: none
  const double *ssrc[SS];    // node-scalar pieces (at chunk start 0)
  int sdst[SS];
  int sgl[SS];               // node of each piece within the chunk

  __device__ __forceinline__ void init(const ClassDesc &D, int N,
                                       const double *__restrict__ T,
                                       const double *__restrict__ S,
                                       const double *__restrict__ Wg,
                                       int lane) {
#pragma unroll
    for (int j = 0; j < SL_MAX; ++j) {
      const int q = lane + 32 * j;
      dst[j] = -1;
      src[j] = T;
      stride[j] = 0;
      if (q < D.nb * 5) {
        const int a = q / 5;
        const int p = q - 5 * a;
        int ia, n;
        member(D, a, ia, n);
        src[j] = (p < 4) ? T + (int64_t)(n - 1) * TMX_NQ + 2 * p
                         : Wg + (int64_t)(n - 1) * 2;
        stride[j] = (p < 4) ? N * TMX_NQ : 2 * N;
        dst[j] = a * TMX_ROW + 2 * p;
      }
    }
#pragma unroll
    for (int j = 0; j < SS; ++j) {
      const int q = lane + 32 * j;
      const int gl = q / (TMX_NS / 2);
      const int p = q - gl * (TMX_NS / 2);
      ssrc[j] = S + (int64_t)gl * TMX_NS + 2 * p;
      sdst[j] = TMX_WG * NBM * TMX_ROW + gl * TMX_NS + 2 * p;
      sgl[j] = gl;
    }
  }

  // copies of nodes [g0, g0 + TMX_WG) (one commit group per lane)
  __device__ __forceinline__ void issue(double *st, int g0, int ng) const {
#pragma unroll
    for (int j = 0; j < SL_MAX; ++j) {
      if (dst[j] >= 0) {
        const double *sp = src[j] + (int64_t)g0 * stride[j];
#pragma unroll
        for (int gl = 0; gl < TMX_WG; ++gl) {
          if (g0 + gl < ng) {
            cp16(st + dst[j] + gl * NBM * TMX_ROW, sp);
          }
          sp += stride[j];
        }
      }
    }
#pragma unroll
    for (int j = 0; j < SS; ++j) {
      if (g0 + sgl[j] < ng) {
        cp16(st + sdst[j], ssrc[j] + (int64_t)g0 * TMX_NS);
      }
    }
    cp_commit();
  }
};

// D += A B for one m8n8k4 FP64 tensor-core tile: lane l holds A[l / 4][l % 4],
// B[l % 4][l / 4] and D[l / 4][2 (l % 4) + {0, 1}]
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, "
      "{%0, %1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// ------------------------------------------ LU and solves in registers --
//
// Row r of a class matrix lives in the registers of the C lanes
// [C r, C r + C) of a warp: lane c of the group holds the columns
// k = c + C t (t < NBM / C). Both routines perform the operations of the
// one-row-per-lane versions in the same order.

// Pivot of one elimination step: the candidate with the largest key (the
// bits of |Q_ri| with the top bit set, which order like the non-negative
// doubles; 0 for lanes that are no candidate), ties to the smallest position.
__device__ __forceinline__ void warp_argmax(unsigned long long key, int pos,
                                            int &best_pos, int &best_lane) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
  const unsigned ml = __reduce_max_sync(0xffffffffu, (hi == mh) ? lo : 0u);
  const bool top = (hi == mh) && (lo == ml) && key != 0ull;
  const unsigned mp = __reduce_min_sync(0xffffffffu, top ? (unsigned)pos : 0xffffffffu);
  const unsigned bal = __ballot_sync(0xffffffffu, top && (unsigned)pos == mp);
  best_pos = (int)mp;
  best_lane = __ffs(bal) - 1;
}

// In-place LU with partial pivoting of the nb x nb matrix Q (row stride LD,
// shared memory) by one warp: the pivot of step i is the first row (by
// position) at or below i with the largest |Q_ri| (Matrix::plu_inverse,
// src/Matrix.hpp:261-384); rows stay in their lanes and carry a position.
// prow: NBM complex of scratch. Returns true if a pivot was zero.
template <int NBM, int C>
__device__ __forceinline__ bool lu_rows(cplx *Qm, int LD, cplx *prow, int *piv,
                                        int nb, int lane) {
  constexpr int NT = NBM / C;
  const int row = lane / C;
  const int c = lane % C;
  cplx q[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    const int k = c + C * t;
    q[t] = (row < nb && k < nb) ? Qm[row * LD + k] : mkc(0., 0.);
  }
  int pos = row;
  bool singular = false;
#pragma unroll
  for (int i = 0; i < NBM; ++i) {
    if (i >= nb) {
      break;
    }
    const bool own = (c == i % C);
    double av = 0.;
    unsigned long long key = 0ull;
    if (own && row < nb && pos >= i) {
      av = cabs_dev(q[i / C]);
      key = (unsigned long long)__double_as_longlong(av) | (1ull << 63);
    }
    int bi, wl;
    warp_argmax(key, pos, bi, wl);
    const double best = __shfl_sync(0xffffffffu, av, wl);
    singular = singular || !(best > 0.);
    if (lane == 0) {
      piv[i] = bi;
    }
    const int wrow = wl / C;
    if (pos == i) {
      pos = bi;
    }
    if (row == wrow) {
      pos = i;
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const int k = c + C * t;
        if (k >= i && k < nb) {
          prow[k] = q[t];
        }
      }
    }
    __syncwarp();
    const bool elim = row < nb && pos > i;
    cplx l = mkc(0., 0.);
    if (elim && own) {
      const cplx pinv = cinv_lu(prow[i]);
      l = cmul(q[i / C], pinv);
      q[i / C] = l;
    }
    l.x = __shfl_sync(0xffffffffu, l.x, i % C, C);
    l.y = __shfl_sync(0xffffffffu, l.y, i % C, C);
    if (elim) {
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const int k = c + C * t;
        if (k > i && k < nb) {
          q[t] = csub(q[t], cmul(l, prow[k]));
        }
      }
    }
    __syncwarp();
  }
  if (row < nb) {
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int k = c + C * t;
      if (k < nb) {
        Qm[pos * LD + k] = q[t];
      }
    }
  }
  return singular;
}

template <int TR, int TC, int MINB, bool MMA>
__global__ void __launch_bounds__(128, MINB)
    k_blocks_warp(TmxBlockArgs A) {
  constexpr int NBM = MMA ? 16 : ((8 * TR > 4 * TC) ? 8 * TR : 4 * TC);
  // row padding unit of the class rows: a tensor row tile of 8 holds one
  // row group only
  constexpr int PR = MMA ? 8 : TR;
  constexpr int LD = NBM + 1;
  static_assert(2 * NBM * LD + 2 * NBM <= warp_elems<NBM>(), "warp smem");
  extern __shared__ __align__(16) unsigned char tmx_wsmem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  cplx *base = reinterpret_cast<cplx *>(tmx_wsmem) + wib * warp_elems<NBM>();
  cplx *Fs = base;                      // [WG][4][NBM]
  cplx *Ws = Fs + TMX_WG * 4 * NBM;     // [2][WG][4][NBM]
  cplx *Qm = base;                      // [NBM][LD]  (after the assembly)
  cplx *Rm = Qm + NBM * LD;             // [NBM][LD]
  cplx *uinv = Rm + NBM * LD;           // [NBM]
  int *perm = reinterpret_cast<int *>(uinv + NBM); // [NBM]
  int *piv = perm + NBM;                           // [NBM]
  double *stg = reinterpret_cast<double *>(
      reinterpret_cast<cplx *>(tmx_wsmem) + 4 * warp_elems<NBM>() +
      wib * warp_stage_elems<NBM>());
  const double *stgS = stg + TMX_WG * NBM * TMX_ROW;
  const int rt = lane >> 2;
  const int ct = lane & 3;
  const int ilo = A.range ? A.range[0] : 0;
  const int ihi = A.range ? min(A.range[1], A.nitems) : A.nitems;
  for (int it = ilo + blockIdx.x * 4 + wib; it < ihi; it += gridDim.x * 4) {
    const TmxItem item = A.items[it];
    const TmxSlot sl = A.slots[item.slot];
    const TmxGrain Gr = A.grains[sl.grain];
    const int N = sl.nmax;
    const int ng = sl.ngauss;
    const int m = item.m;
    const ClassDesc D = describe<PR>(N, m, item.cls);
    const int nb = D.nb;
    if (nb <= 0) {
      continue;
    }
    if (nb > NBM || D.NRp > NBM) {
      if (lane == 0) {
        atomicOr(&A.status[sl.grain], TMX_ST_TOO_LARGE);
      }
      continue;
    }
    const double *T = A.tab + sl.tab;
    const double *S = A.nsc + sl.nsc;
    const double *Wg = A.wig + A.wig_off[sl.wig_n] + (int64_t)m * ng * N * 2;
    const double k2 = Gr.k * Gr.k;
    const cplx k2mr = mkc(Gr.mr * k2, Gr.mi * k2);
    const int ngroups = (D.R1 > 0 && m > 0) ? 2 : 1;

    // ---------------------------------------------------------- assembly
    // DFMA path: aj/ay[TR][TC]; tensor path: acc[row tile][col tile][jr, ji,
    // yr, yi] as m8n8 accumulator fragments
    double aj[TR][TC][2], ay[TR][TC][2];
    double acc[2][2][4][2];
#pragma unroll
    for (int r = 0; r < TR; ++r) {
#pragma unroll
      for (int c = 0; c < TC; ++c) {
        aj[r][c][0] = aj[r][c][1] = ay[r][c][0] = ay[r][c][1] = 0.;
      }
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          acc[r][c][p][0] = acc[r][c][p][1] = 0.;
        }
      }
    }
    // rows are padded per group to a multiple of TR (describe<TR>), so the
    // TR rows of a lane share one row group and one set of B-side vectors
    const int rgl = (rt * TR < D.R0p) ? 0 : 1;
    // the table rows of each chunk are staged in shared memory while the
    // previous chunk is contracted
    StagePlan<NBM> plan;
    plan.init(D, N, T, S, Wg, lane);
    plan.issue(stg, 0, ng);
    for (int g0 = 0; g0 < ng; g0 += TMX_WG) {
      cp_wait_all();
      __syncwarp();
      // slots (node gl, row or column) = (u / NBM, u % NBM): TMX_WG NBM / 32
      // per lane on each side, unrolled so that their shared-memory reads and
      // arithmetic interleave
      constexpr int NIT = TMX_WG * NBM / 32;
      static_assert(NIT * 32 == TMX_WG * NBM, "build slots");
#pragma unroll
      for (int j = 0; j < NIT; ++j) {
        const int u = lane + 32 * j;
        const int gl = u / NBM;
        const int pr = u % NBM;
        if (pr >= D.NRp) {
          continue;
        }
        const int a = padded_member(D, pr);
        cplx *fp = Fs + gl * 4 * NBM + pr;
        if (a >= 0 && g0 + gl < ng) {
          int ia, n;
          member(D, a, ia, n);
          const double *r = stg + (gl * NBM + a) * TMX_ROW;
          const double2 jd = *reinterpret_cast<const double2 *>(r + TMX_Q_J);
          const double2 yd = *reinterpret_cast<const double2 *>(r + TMX_Q_Y);
          const double2 wd = *reinterpret_cast<const double2 *>(r + TMX_NQ);
          a_side_row<true>(jd.x, jd.y, yd.x, yd.y, wd.x, wd.y, stgS + gl * TMX_NS,
                           n, fp, NBM, m);
        } else {
          zero_side(fp, NBM, 4);
        }
      }
#pragma unroll
      for (int j = 0; j < NIT; ++j) {
        const int u = lane + 32 * j;
        const int gl = u / NBM;
        const int b = u % NBM;
        if (b >= nb) {
          continue;
        }
        cplx *wp = Ws + gl * 4 * NBM + b;
        if (g0 + gl < ng) {
          int ib, n;
          member(D, b, ib, n);
          const double *r = stg + (gl * NBM + b) * TMX_ROW;
          const double2 jm = *reinterpret_cast<const double2 *>(r + TMX_Q_JM_RE);
          const double2 djm = *reinterpret_cast<const double2 *>(r + TMX_Q_DJM_RE);
          const double2 wd = *reinterpret_cast<const double2 *>(r + TMX_NQ);
          b_side_row<true>(D, ib, n, m, jm, djm, wd.x, wd.y, stgS + gl * TMX_NS,
                           ngroups, k2, k2mr, wp, NBM, TMX_WG * 4 * NBM);
        } else {
          for (int q = 0; q < ngroups; ++q) {
            zero_side(wp + q * TMX_WG * 4 * NBM, NBM, 4);
          }
        }
      }
      __syncwarp();
      if (g0 + TMX_WG < ng) {
        plan.issue(stg, g0 + TMX_WG, ng);
      }
      const int gmax = min(TMX_WG, ng - g0);
      if constexpr (MMA) {
        // K slices of 4: the four terms of one node (m >= 1), or terms 1 and
        // 3 of two nodes (m = 0, where terms 0 and 2 vanish)
        // padded row tile rti holds row group (rti * 8 < R0p ? 0 : 1) only
        const int q = lane & 3;
        const int rr = lane >> 2;
        const int nrt = D.NRp >> 3;
        const int nct = (nb + 7) >> 3;
        const int nsl = (m == 0) ? (gmax + 1) >> 1 : gmax;
        for (int sx = 0; sx < nsl; ++sx) {
          const int gl = (m == 0) ? 2 * sx + (q >> 1) : sx;
          const int t = (m == 0) ? 1 + 2 * (q & 1) : q;
#pragma unroll
          for (int rti = 0; rti < 2; ++rti) {
            if (rti < nrt) {
              const cplx f = Fs[(gl * 4 + t) * NBM + rti * 8 + rr];
              const int g = (rti * 8 < D.R0p) ? 0 : 1;
#pragma unroll
              for (int cti = 0; cti < 2; ++cti) {
                if (cti < nct) {
                  const int col = cti * 8 + rr;
                  const cplx w = (col < nb)
                      ? Ws[((g * TMX_WG + gl) * 4 + t) * NBM + col]
                      : mkc(0., 0.);
                  double *a4 = &acc[rti][cti][0][0];
                  dmma(a4[0], a4[1], f.x, w.x); // jr
                  dmma(a4[2], a4[3], f.x, w.y); // ji
                  dmma(a4[4], a4[5], f.y, w.x); // yr
                  dmma(a4[6], a4[7], f.y, w.y); // yi
                }
              }
            }
          }
        }
      } else {
        // one term t of node gl; the terms of a node are unrolled (t = 1, 3
        // for m = 0, where mu = 0 removes t = 0, 2) so their reads overlap
        auto term = [&](int gl, int t) {
          const cplx *fr = Fs + (gl * 4 + t) * NBM + rt * TR;
          const cplx *wr = Ws + (rgl * TMX_WG * 4 + gl * 4 + t) * NBM + ct;
          cplx w[TC];
#pragma unroll
          for (int c = 0; c < TC; ++c) {
            w[c] = wr[4 * c];
          }
#pragma unroll
          for (int r = 0; r < TR; ++r) {
            const cplx f = fr[r];
#pragma unroll
            for (int c = 0; c < TC; ++c) {
              aj[r][c][0] = fma(f.x, w[c].x, aj[r][c][0]);
              aj[r][c][1] = fma(f.x, w[c].y, aj[r][c][1]);
              ay[r][c][0] = fma(f.y, w[c].x, ay[r][c][0]);
              ay[r][c][1] = fma(f.y, w[c].y, ay[r][c][1]);
            }
          }
        };
        if (m == 0) {
          for (int gl = 0; gl < gmax; ++gl) {
            term(gl, 1);
            term(gl, 3);
          }
        } else {
          for (int gl = 0; gl < gmax; ++gl) {
#pragma unroll
            for (int t = 0; t < 4; ++t) {
              term(gl, t);
            }
          }
        }
      }
    }
    __syncwarp();
    // a_n of each member once per item (in the 1/U_jj slots, free until the
    // LU); entry (a, b) is scaled by a_n(n_a) a_n(n_b)
    double *an_s = reinterpret_cast<double *>(uinv);
    if (lane < nb) {
      int ia, na;
      member(D, lane, ia, na);
      an_s[lane] = a_n(na);
    }
    __syncwarp();
    // Q = G^j + i G^y, RgQ = G^j, into the (reused) chunk buffers
    if constexpr (MMA) {
      const int rr = lane >> 2;
      const int q = lane & 3;
#pragma unroll
      for (int rti = 0; rti < 2; ++rti) {
#pragma unroll
        for (int cti = 0; cti < 2; ++cti) {
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int a = padded_member(D, rti * 8 + rr);
            const int b = cti * 8 + 2 * q + i;
            if (a >= 0 && b < nb) {
              const double sc = an_s[a] * an_s[b];
              const double jr = acc[rti][cti][0][i], ji = acc[rti][cti][1][i];
              const double yr = acc[rti][cti][2][i], yi = acc[rti][cti][3][i];
              Qm[a * LD + b] = mkc((jr - yi) * sc, (ji + yr) * sc);
              Rm[a * LD + b] = mkc(jr * sc, ji * sc);
            }
          }
        }
      }
    } else {
#pragma unroll
      for (int r = 0; r < TR; ++r) {
        const int a = padded_member(D, rt * TR + r);
#pragma unroll
        for (int c = 0; c < TC; ++c) {
          const int b = ct + 4 * c;
          if (a >= 0 && b < nb) {
            const double sc = an_s[a] * an_s[b];
            Qm[a * LD + b] = mkc((aj[r][c][0] - ay[r][c][1]) * sc,
                                 (aj[r][c][1] + ay[r][c][0]) * sc);
            Rm[a * LD + b] = mkc(aj[r][c][0] * sc, aj[r][c][1] * sc);
          }
        }
      }
    }
    __syncwarp();

    // ---------------------------------------------------------------- LU
    // in registers, 32 / NBM lanes per row; the pivot row goes through uinv
    constexpr int CL = 32 / NBM;
    const bool singular = lu_rows<NBM, CL>(Qm, LD, uinv, piv, nb, lane);
    __syncwarp();
    if (lane < nb) {
      uinv[lane] = cinv_lu(Qm[lane * LD + lane]);
    }
    if (lane == 0) {
      // column exchanges of Matrix::plu_inverse step 4, as a gather index
      for (int j = 0; j < nb; ++j) {
        perm[j] = j;
      }
      for (int j = nb - 1; j >= 0; --j) {
        const int p = piv[j];
        const int t = perm[j];
        perm[j] = perm[p];
        perm[p] = t;
      }
      if (singular) {
        atomicOr(&A.status[sl.grain], TMX_ST_SINGULAR);
      }
    }
    __syncwarp();
    if (A.lu) {
      cplx *Ls = A.lu + item.scratch;
      for (int u = lane; u < nb * nb; u += 32) {
        Ls[u] = Qm[(u / nb) * LD + (u % nb)];
      }
      int *ps = reinterpret_cast<int *>(Ls + (int64_t)nb * nb);
      for (int j = lane; j < nb; j += 32) {
        ps[j] = perm[j];
      }
    }

    // ------------------------------------------ solve T_c Q_c = -RgQ_c
    solve_rows<NBM, CL>(Rm, Qm, LD, uinv, nb, lane / CL, lane % CL);
    __syncwarp();
    // write out: T_c[a][b] = Y[a][perm[b]]
    if (sl.tout < 0) {
      if (lane < nb) {
        int ia, na;
        member(D, lane, ia, na);
        A.diag[sl.diag + ia * N + (na - 1)] = Rm[lane * LD + perm[lane]];
      }
    } else {
      cplx *Tb = A.tout + sl.tout + block_offset(N, m);
      const int w2 = 2 * D.nbb;
      for (int u = lane; u < nb * nb; u += 32) {
        const int a = u / nb;
        const int b = u - a * nb;
        int ia, na, ib, nbn;
        member(D, a, ia, na);
        member(D, b, ib, nbn);
        const int rowi = ia * D.nbb + (na - D.nmin);
        const int col = ib * D.nbb + (nbn - D.nmin);
        Tb[(int64_t)rowi * w2 + col] = Rm[a * LD + perm[b]];
      }
    }
    __syncwarp();
  }
}

template <int TR, int TC, int MINB, bool MMA>
static void launch_warp_variant(const TmxBlockArgs &a, cudaStream_t stream) {
  constexpr int NBM = MMA ? 16 : ((8 * TR > 4 * TC) ? 8 * TR : 4 * TC);
  const size_t smem =
      (size_t)4 * (warp_elems<NBM>() + warp_stage_elems<NBM>()) * sizeof(cplx);
  cudaFuncSetAttribute(k_blocks_warp<TR, TC, MINB, MMA>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  // one item per warp: CTAs retire after one item, so that launches of the
  // high-priority order loop get SMs between them (a grid of long-lived
  // CTAs looping over items held the SMs for a whole round)
  int blocks = (int)std::max<int64_t>(1, ((int64_t)a.nitems + 3) / 4);
  if (a.max_ctas > 0) {
    blocks = std::min(blocks, a.max_ctas);
  }
  k_blocks_warp<TR, TC, MINB, MMA><<<blocks, 128, smem, stream>>>(a);
}

// ------------------------------------------ four warps per item (<= 32) --
//
// Classes of 17..32 members: one CTA of four warps per item. The warps
// build each chunk of TMX_WG32 nodes together (one barrier), warp w then
// accumulates column tile w (columns 8w..8w+7) over all four row tiles on
// the FP64 tensor pipe (as in k_blocks_warp's tensor path), and warp 0
// factors and solves with one lane per row (no barriers inside the LU).

#define TMX_WG32 4

__host__ __device__ constexpr int cta32_elems() {
  // F[WG][4][32] + W[2][WG][4][32], or Q, RgQ [32][33], 1/U_jj, indices
  return (12 * TMX_WG32 * 32 > 2 * 32 * 33 + 3 * 32) ? 12 * TMX_WG32 * 32
                                                      : 2 * 32 * 33 + 3 * 32;
}

__global__ void __launch_bounds__(128, 4) k_blocks_cta32(TmxBlockArgs A) {
  constexpr int NBM = 32;
  constexpr int LD = NBM + 1;
  extern __shared__ __align__(16) unsigned char tmx_c32smem[];
  cplx *base = reinterpret_cast<cplx *>(tmx_c32smem);
  cplx *Fs = base;                   // [WG][4][NBM]
  cplx *Ws = Fs + TMX_WG32 * 4 * NBM; // [2][WG][4][NBM]
  cplx *Qm = base;                   // [NBM][LD]  (after the assembly)
  cplx *Rm = Qm + NBM * LD;          // [NBM][LD]
  cplx *uinv = Rm + NBM * LD;        // [NBM]
  int *perm = reinterpret_cast<int *>(uinv + NBM); // [NBM]
  int *piv = perm + NBM;                           // [NBM]
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wib = tid >> 5;
  const int q = lane & 3;
  const int rr = lane >> 2;
  const int ilo = A.range ? A.range[0] : 0;
  const int ihi = A.range ? min(A.range[1], A.nitems) : A.nitems;
  for (int it = ilo + blockIdx.x; it < ihi; it += gridDim.x) {
    const TmxItem item = A.items[it];
    const TmxSlot sl = A.slots[item.slot];
    const TmxGrain Gr = A.grains[sl.grain];
    const int N = sl.nmax;
    const int ng = sl.ngauss;
    const int m = item.m;
    const ClassDesc D = describe<1>(N, m, item.cls);
    const int nb = D.nb;
    if (nb <= 0) {
      continue;
    }
    if (nb > NBM) {
      if (tid == 0) {
        atomicOr(&A.status[sl.grain], TMX_ST_TOO_LARGE);
      }
      continue;
    }
    const double *T = A.tab + sl.tab;
    const double *S = A.nsc + sl.nsc;
    const double *Wg = A.wig + A.wig_off[sl.wig_n] + (int64_t)m * ng * N * 2;
    const double k2 = Gr.k * Gr.k;
    const cplx k2mr = mkc(Gr.mr * k2, Gr.mi * k2);
    const int ngroups = (D.R1 > 0 && m > 0) ? 2 : 1;
    const int nrt = (nb + 7) >> 3;
    const int col = wib * 8 + rr; // B-fragment column of this lane
    double acc[4][4][2];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        acc[r][p][0] = acc[r][p][1] = 0.;
      }
    }
    for (int g0 = 0; g0 < ng; g0 += TMX_WG32) {
      __syncthreads();
      for (int u = tid; u < TMX_WG32 * nb; u += 128) {
        const int gl = u / nb;
        const int a = u - gl * nb;
        cplx *fp = Fs + gl * 4 * NBM + a;
        cplx *wp = Ws + gl * 4 * NBM + a;
        if (g0 + gl < ng) {
          a_side<true>(D, a, N, g0 + gl, T, S, Wg, fp, NBM, m);
          b_side<true>(D, a, N, m, g0 + gl, ngroups, T, S, Wg, k2, k2mr, wp, NBM,
                       TMX_WG32 * 4 * NBM);
        } else {
          zero_side(fp, NBM, 4);
          for (int g = 0; g < ngroups; ++g) {
            zero_side(wp + g * TMX_WG32 * 4 * NBM, NBM, 4);
          }
        }
      }
      __syncthreads();
      if (wib * 8 < nb) {
        const int gmax = min(TMX_WG32, ng - g0);
        const int nsl = (m == 0) ? (gmax + 1) >> 1 : gmax;
        for (int sx = 0; sx < nsl; ++sx) {
          const int gl = (m == 0) ? 2 * sx + (q >> 1) : sx;
          const int t = (m == 0) ? 1 + 2 * (q & 1) : q;
          cplx w[2];
#pragma unroll
          for (int g = 0; g < 2; ++g) {
            w[g] = (col < nb && g < ngroups)
                       ? Ws[((g * TMX_WG32 + gl) * 4 + t) * NBM + col]
                       : mkc(0., 0.);
          }
#pragma unroll
          for (int rti = 0; rti < 4; ++rti) {
            if (rti < nrt) {
              const int row = rti * 8 + rr;
              const cplx f = (row < nb) ? Fs[(gl * 4 + t) * NBM + row] : mkc(0., 0.);
              const int grp = (row < D.R0) ? 0 : 1;
              const int lo = rti * 8, hi = min(rti * 8 + 8, nb);
#pragma unroll
              for (int g = 0; g < 2; ++g) {
                const bool present = (g == 0) ? (lo < D.R0) : (ngroups == 2 && hi > D.R0);
                if (present) {
                  const double fj = (grp == g) ? f.x : 0.;
                  const double fy = (grp == g) ? f.y : 0.;
                  double *a4 = &acc[rti][0][0];
                  dmma(a4[0], a4[1], fj, w[g].x);
                  dmma(a4[2], a4[3], fj, w[g].y);
                  dmma(a4[4], a4[5], fy, w[g].x);
                  dmma(a4[6], a4[7], fy, w[g].y);
                }
              }
            }
          }
        }
      }
    }
    // a_n of each member once per item (in the 1/U_jj slots, free until the
    // LU)
    double *an_s = reinterpret_cast<double *>(uinv);
    if (tid < nb) {
      int ia, na;
      member(D, tid, ia, na);
      an_s[tid] = a_n(na);
    }
    __syncthreads();
    // Q = G^j + i G^y, RgQ = G^j (times a_n1 a_n2), into the chunk buffers
#pragma unroll
    for (int rti = 0; rti < 4; ++rti) {
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int a = rti * 8 + rr;
        const int b = wib * 8 + 2 * q + i;
        if (a < nb && b < nb) {
          const double sc = an_s[a] * an_s[b];
          const double jr = acc[rti][0][i], ji = acc[rti][1][i];
          const double yr = acc[rti][2][i], yi = acc[rti][3][i];
          Qm[a * LD + b] = mkc((jr - yi) * sc, (ji + yr) * sc);
          Rm[a * LD + b] = mkc(jr * sc, ji * sc);
        }
      }
    }
    // every warp's column tiles of Q are in place before warp 0 factors
    __syncthreads();
    if (wib == 0) {
      // LU in place in Qm, lane r updates row r
      bool singular = false;
      for (int i = 0; i < nb; ++i) {
        double best = (lane >= i && lane < nb) ? cabs_dev(Qm[lane * LD + i]) : -1.;
        int bi = lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double ov = __shfl_xor_sync(0xffffffffu, best, o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
          if (ov > best || (ov == best && oi < bi)) {
            best = ov;
            bi = oi;
          }
        }
        singular = singular || !(best > 0.);
        if (lane == 0) {
          piv[i] = bi;
        }
        if (bi != i) {
          for (int k = lane; k < nb; k += 32) {
            const cplx t = Qm[i * LD + k];
            Qm[i * LD + k] = Qm[bi * LD + k];
            Qm[bi * LD + k] = t;
          }
        }
        __syncwarp();
        if (lane > i && lane < nb) {
          const cplx pinv = cinv_lu(Qm[i * LD + i]);
          const cplx l = cmul(Qm[lane * LD + i], pinv);
          Qm[lane * LD + i] = l;
          // four entries at a time: all loads before the stores (the pivot
          // row is only read in this step), so the updates overlap
          cplx *qr = Qm + lane * LD;
          const cplx *pr = Qm + i * LD;
          int k = i + 1;
          for (; k + 3 < nb; k += 4) {
            cplx a0 = qr[k], a1 = qr[k + 1], a2 = qr[k + 2], a3 = qr[k + 3];
            const cplx b0 = pr[k], b1 = pr[k + 1], b2 = pr[k + 2], b3 = pr[k + 3];
            a0 = csub(a0, cmul(l, b0));
            a1 = csub(a1, cmul(l, b1));
            a2 = csub(a2, cmul(l, b2));
            a3 = csub(a3, cmul(l, b3));
            qr[k] = a0;
            qr[k + 1] = a1;
            qr[k + 2] = a2;
            qr[k + 3] = a3;
          }
          for (; k < nb; ++k) {
            qr[k] = csub(qr[k], cmul(l, pr[k]));
          }
        }
        __syncwarp();
      }
      if (lane < nb) {
        uinv[lane] = cinv_lu(Qm[lane * LD + lane]);
      }
      if (lane == 0) {
        // column exchanges of Matrix::plu_inverse step 4, as a gather index
        for (int j = 0; j < nb; ++j) {
          perm[j] = j;
        }
        for (int j = nb - 1; j >= 0; --j) {
          const int p = piv[j];
          const int t = perm[j];
          perm[j] = perm[p];
          perm[p] = t;
        }
        if (singular) {
          atomicOr(&A.status[sl.grain], TMX_ST_SINGULAR);
        }
      }
    }
    __syncthreads();
    // solve T_c Q_c = -RgQ_c: four lanes per row, row 8 w + lane / 4
    solve_rows<NBM, 4>(Rm, Qm, LD, uinv, nb, wib * 8 + (lane >> 2), lane & 3);
    __syncthreads();
    if (A.lu) {
      cplx *Ls = A.lu + item.scratch;
      for (int u = tid; u < nb * nb; u += 128) {
        Ls[u] = Qm[(u / nb) * LD + (u % nb)];
      }
      int *ps = reinterpret_cast<int *>(Ls + (int64_t)nb * nb);
      for (int j = tid; j < nb; j += 128) {
        ps[j] = perm[j];
      }
    }
    // write out: T_c[a][b] = Y[a][perm[b]]
    if (sl.tout < 0) {
      if (tid < nb) {
        int ia, na;
        member(D, tid, ia, na);
        A.diag[sl.diag + ia * N + (na - 1)] = Rm[tid * LD + perm[tid]];
      }
    } else {
      cplx *Tb = A.tout + sl.tout + block_offset(N, m);
      const int w2 = 2 * D.nbb;
      for (int u = tid; u < nb * nb; u += 128) {
        const int a = u / nb;
        const int b = u - a * nb;
        int ia, na, ib, nbn;
        member(D, a, ia, na);
        member(D, b, ib, nbn);
        Tb[(int64_t)(ia * D.nbb + (na - D.nmin)) * w2 + ib * D.nbb + (nbn - D.nmin)] =
            Rm[a * LD + perm[b]];
      }
    }
  }
}

// ------------------------------------------ eight warps per item (<= 64) --
//
// Classes of 33..64 members: one CTA of eight warps per item. As in
// k_blocks_cta32 the warps build each chunk of TMX_WG32 nodes together and
// warp w accumulates column tile w over all eight row tiles with DMMA, so
// the node factors are built once per item; the LU pivots with warp 0 and
// updates with all threads (four barriers per step), and the solves keep
// each row in the registers of four lanes (row tid / 4).

__host__ __device__ constexpr int cta64_elems() {
  // F[WG][4][64] + W[2][WG][4][64], or Q, RgQ [64][65], 1/U_jj, pivot and
  // gather indices and a flag
  return (12 * TMX_WG32 * 64 > 2 * 64 * 65 + 64 + 66) ? 12 * TMX_WG32 * 64
                                                        : 2 * 64 * 65 + 64 + 66;
}

__global__ void __launch_bounds__(256, 1) k_blocks_cta64(TmxBlockArgs A) {
  constexpr int NBM = 64;
  constexpr int LD = NBM + 1;
  constexpr int NTH = 256;
  extern __shared__ __align__(16) unsigned char tmx_c64smem[];
  cplx *base = reinterpret_cast<cplx *>(tmx_c64smem);
  cplx *Fs = base;                    // [WG][4][NBM]
  cplx *Ws = Fs + TMX_WG32 * 4 * NBM; // [2][WG][4][NBM]
  cplx *Qm = base;                    // [NBM][LD]  (after the assembly)
  cplx *Rm = Qm + NBM * LD;           // [NBM][LD]
  cplx *uinv = Rm + NBM * LD;         // [NBM]
  int *perm = reinterpret_cast<int *>(uinv + NBM); // [NBM]
  int *piv = perm + NBM;                           // [NBM]
  int *flag = piv + NBM;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wib = tid >> 5;
  const int q = lane & 3;
  const int rr = lane >> 2;
  const int ilo = A.range ? A.range[0] : 0;
  const int ihi = A.range ? min(A.range[1], A.nitems) : A.nitems;
  for (int it = ilo + blockIdx.x; it < ihi; it += gridDim.x) {
    const TmxItem item = A.items[it];
    const TmxSlot sl = A.slots[item.slot];
    const TmxGrain Gr = A.grains[sl.grain];
    const int N = sl.nmax;
    const int ng = sl.ngauss;
    const int m = item.m;
    const ClassDesc D = describe<1>(N, m, item.cls);
    const int nb = D.nb;
    if (nb <= 0) {
      continue;
    }
    if (nb > NBM) {
      if (tid == 0) {
        atomicOr(&A.status[sl.grain], TMX_ST_TOO_LARGE);
      }
      continue;
    }
    const double *T = A.tab + sl.tab;
    const double *S = A.nsc + sl.nsc;
    const double *Wg = A.wig + A.wig_off[sl.wig_n] + (int64_t)m * ng * N * 2;
    const double k2 = Gr.k * Gr.k;
    const cplx k2mr = mkc(Gr.mr * k2, Gr.mi * k2);
    const int ngroups = (D.R1 > 0 && m > 0) ? 2 : 1;
    const int nrt = (nb + 7) >> 3;
    const int col = wib * 8 + rr; // B-fragment column of this lane
    double acc[8][4][2];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        acc[r][p][0] = acc[r][p][1] = 0.;
      }
    }
    for (int g0 = 0; g0 < ng; g0 += TMX_WG32) {
      __syncthreads();
      for (int u = tid; u < TMX_WG32 * nb; u += NTH) {
        const int gl = u / nb;
        const int a = u - gl * nb;
        cplx *fp = Fs + gl * 4 * NBM + a;
        cplx *wp = Ws + gl * 4 * NBM + a;
        if (g0 + gl < ng) {
          a_side<true>(D, a, N, g0 + gl, T, S, Wg, fp, NBM, m);
          b_side<true>(D, a, N, m, g0 + gl, ngroups, T, S, Wg, k2, k2mr, wp, NBM,
                       TMX_WG32 * 4 * NBM);
        } else {
          zero_side(fp, NBM, 4);
          for (int g = 0; g < ngroups; ++g) {
            zero_side(wp + g * TMX_WG32 * 4 * NBM, NBM, 4);
          }
        }
      }
      __syncthreads();
      if (wib * 8 < nb) {
        const int gmax = min(TMX_WG32, ng - g0);
        const int nsl = (m == 0) ? (gmax + 1) >> 1 : gmax;
        for (int sx = 0; sx < nsl; ++sx) {
          const int gl = (m == 0) ? 2 * sx + (q >> 1) : sx;
          const int t = (m == 0) ? 1 + 2 * (q & 1) : q;
          cplx w[2];
#pragma unroll
          for (int g = 0; g < 2; ++g) {
            w[g] = (col < nb && g < ngroups)
                       ? Ws[((g * TMX_WG32 + gl) * 4 + t) * NBM + col]
                       : mkc(0., 0.);
          }
#pragma unroll
          for (int rti = 0; rti < 8; ++rti) {
            if (rti < nrt) {
              const int row = rti * 8 + rr;
              const cplx f = (row < nb) ? Fs[(gl * 4 + t) * NBM + row] : mkc(0., 0.);
              const int grp = (row < D.R0) ? 0 : 1;
              const int lo = rti * 8, hi = min(rti * 8 + 8, nb);
#pragma unroll
              for (int g = 0; g < 2; ++g) {
                const bool present = (g == 0) ? (lo < D.R0) : (ngroups == 2 && hi > D.R0);
                if (present) {
                  const double fj = (grp == g) ? f.x : 0.;
                  const double fy = (grp == g) ? f.y : 0.;
                  double *a4 = &acc[rti][0][0];
                  dmma(a4[0], a4[1], fj, w[g].x);
                  dmma(a4[2], a4[3], fj, w[g].y);
                  dmma(a4[4], a4[5], fy, w[g].x);
                  dmma(a4[6], a4[7], fy, w[g].y);
                }
              }
            }
          }
        }
      }
    }
    // a_n of each member once per item (in the 1/U_jj slots)
    double *an_s = reinterpret_cast<double *>(uinv);
    if (tid < nb) {
      int ia, na;
      member(D, tid, ia, na);
      an_s[tid] = a_n(na);
    }
    if (tid == 0) {
      *flag = 0;
    }
    __syncthreads();
    // Q = G^j + i G^y, RgQ = G^j (times a_n1 a_n2), into the chunk buffers
#pragma unroll
    for (int rti = 0; rti < 8; ++rti) {
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int a = rti * 8 + rr;
        const int b = wib * 8 + 2 * q + i;
        if (a < nb && b < nb) {
          const double sc = an_s[a] * an_s[b];
          const double jr = acc[rti][0][i], ji = acc[rti][1][i];
          const double yr = acc[rti][2][i], yi = acc[rti][3][i];
          Qm[a * LD + b] = mkc((jr - yi) * sc, (ji + yr) * sc);
          Rm[a * LD + b] = mkc(jr * sc, ji * sc);
        }
      }
    }
    __syncthreads();
    // LU in place in Qm: pivot of column i by warp 0 (first row with the
    // largest |Q_ri|), row exchange, column scaling, rank-1 update
    for (int i = 0; i < nb; ++i) {
      if (wib == 0) {
        double best = -1.;
        int bi = i;
        for (int j = i + lane; j < nb; j += 32) {
          const double v = cabs_dev(Qm[j * LD + i]);
          if (v > best) {
            best = v;
            bi = j;
          }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double ov = __shfl_down_sync(0xffffffffu, best, o);
          const int oi = __shfl_down_sync(0xffffffffu, bi, o);
          if (ov > best || (ov == best && oi < bi)) {
            best = ov;
            bi = oi;
          }
        }
        if (lane == 0) {
          piv[i] = bi;
          if (!(best > 0.)) {
            *flag = 1;
          }
        }
      }
      __syncthreads();
      const int ip = piv[i];
      if (ip != i) {
        for (int j = tid; j < nb; j += NTH) {
          const cplx t = Qm[i * LD + j];
          Qm[i * LD + j] = Qm[ip * LD + j];
          Qm[ip * LD + j] = t;
        }
        __syncthreads();
      }
      const cplx pinv = cinv_lu(Qm[i * LD + i]);
      for (int j = i + 1 + tid; j < nb; j += NTH) {
        Qm[j * LD + i] = cmul(Qm[j * LD + i], pinv);
      }
      __syncthreads();
      const int rem = nb - i - 1;
      for (int u = tid; u < rem * rem; u += NTH) {
        const int j = i + 1 + u / rem;
        const int k = i + 1 + u % rem;
        Qm[j * LD + k] = csub(Qm[j * LD + k], cmul(Qm[j * LD + i], Qm[i * LD + k]));
      }
      __syncthreads();
    }
    for (int j = tid; j < nb; j += NTH) {
      uinv[j] = cinv_lu(Qm[j * LD + j]);
    }
    if (tid == 0) {
      // column exchanges of Matrix::plu_inverse step 4, as a gather index
      for (int j = 0; j < nb; ++j) {
        perm[j] = j;
      }
      for (int j = nb - 1; j >= 0; --j) {
        const int p = piv[j];
        const int t = perm[j];
        perm[j] = perm[p];
        perm[p] = t;
      }
      if (*flag) {
        atomicOr(&A.status[sl.grain], TMX_ST_SINGULAR);
      }
    }
    __syncthreads();
    if (A.lu) {
      cplx *Ls = A.lu + item.scratch;
      for (int u = tid; u < nb * nb; u += NTH) {
        Ls[u] = Qm[(u / nb) * LD + (u % nb)];
      }
      int *ps = reinterpret_cast<int *>(Ls + (int64_t)nb * nb);
      for (int j = tid; j < nb; j += NTH) {
        ps[j] = perm[j];
      }
    }
    // solve T_c Q_c = -RgQ_c: four lanes per row
    solve_rows<NBM, 4>(Rm, Qm, LD, uinv, nb, tid >> 2, tid & 3);
    __syncthreads();
    // write out: T_c[a][b] = Y[a][perm[b]]
    if (sl.tout < 0) {
      for (int a = tid; a < nb; a += NTH) {
        int ia, na;
        member(D, a, ia, na);
        A.diag[sl.diag + ia * N + (na - 1)] = Rm[a * LD + perm[a]];
      }
    } else {
      cplx *Tb = A.tout + sl.tout + block_offset(N, m);
      const int w2 = 2 * D.nbb;
      for (int u = tid; u < nb * nb; u += NTH) {
        const int a = u / nb;
        const int b = u - a * nb;
        int ia, na, ib, nbn;
        member(D, a, ia, na);
        member(D, b, ib, nbn);
        Tb[(int64_t)(ia * D.nbb + (na - D.nmin)) * w2 + ib * D.nbb + (nbn - D.nmin)] =
            Rm[a * LD + perm[b]];
      }
    }
    __syncthreads();
  }
}

static void launch_cta64(const TmxBlockArgs &a, cudaStream_t stream) {
  const size_t smem = (size_t)cta64_elems() * sizeof(cplx);
  cudaFuncSetAttribute(k_blocks_cta64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  // one item per CTA (see launch_warp_variant)
  const int blocks = (a.max_ctas > 0) ? std::min(std::max(1, a.nitems), a.max_ctas)
                                       : std::max(1, a.nitems);
  k_blocks_cta64<<<blocks, 256, smem, stream>>>(a);
}

static void launch_cta32(const TmxBlockArgs &a, cudaStream_t stream) {
  const size_t smem = (size_t)cta32_elems() * sizeof(cplx);
  cudaFuncSetAttribute(k_blocks_cta32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  // one item per CTA (see launch_warp_variant)
  const int blocks = (a.max_ctas > 0) ? std::min(std::max(1, a.nitems), a.max_ctas)
                                       : std::max(1, a.nitems);
  k_blocks_cta32<<<blocks, 128, smem, stream>>>(a);
}

// dynamic shared memory the CTA kernel may use (of the 227 KB per block)
#define TMX_BLOCK_SMEM_MAX (227u * 1024u)

// shared memory of one block: the larger of the assembly chunk buffers and
// the LU phase (factors, pivots and a right-hand-side chunk, or the pivot
// data alone for classes whose factors do not fit)
size_t tmx_block_smem_bytes(int max_nb, int chunk_nodes) {
  const int nrp = (max_nb + 3) / 4 * 4 + 4;
  const int ncol = (max_nb + 3) / 4 * 4;
  const size_t asm_bytes =
      ((size_t)4 * chunk_nodes * nrp + (size_t)2 * 4 * chunk_nodes * ncol) *
      sizeof(cplx);
  const int lda = max_nb | 1;
  size_t lu = ((size_t)max_nb * lda + max_nb) * sizeof(cplx) +
              (3 * max_nb + 1) * sizeof(int);
  lu = (lu + 15) & ~(size_t)15;
  // at least 8 rows of the right-hand side per solve chunk
  const int rows = max_nb < 8 ? max_nb : 8;
  size_t lu_total = lu + (size_t)rows * lda * sizeof(cplx);
  // prefer the whole right-hand side when it fits in 200 KB
  const size_t full = lu + (size_t)max_nb * lda * sizeof(cplx);
  if (full <= 200 * 1024) {
    lu_total = full;
  }
  if (lu_total > TMX_BLOCK_SMEM_MAX) {
    // the kernel factors such classes in global memory: shared memory holds
    // the pivot data only
    lu_total = ((size_t)max_nb * sizeof(cplx) + (3 * max_nb + 1) * sizeof(int) + 15) &
               ~(size_t)15;
  }
  return asm_bytes > lu_total ? asm_bytes : lu_total;
}

template <int TR, int TC, int NT, int MINB>
static void launch_variant(const TmxBlockArgs &a, size_t smem,
                           cudaStream_t stream) {
  static int attr_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaFuncSetAttribute(k_blocks<TR, TC, NT, MINB>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         227 * 1024);
    attr_dev = dev;
  }
  const int blocks = (a.max_ctas > 0) ? std::min(std::max(1, a.nitems), a.max_ctas)
                                       : std::max(1, a.nitems);
  k_blocks<TR, TC, NT, MINB><<<blocks, NT, smem, stream>>>(a, smem);
}

int tmx_block_family_capacity(int family) {
  switch (family) {
  case TMX_BLOCKS_WARP_DFMA:
    return 8;
  case TMX_BLOCKS_WARP_DMMA:
    return 16;
  case TMX_BLOCKS_CTA32:
    return 32;
  case TMX_BLOCKS_CTA64:
    return 64;
  case TMX_BLOCKS_CTA:
    return TMX_MAX_NB;
  default:
    return 0;
  }
}

// The family given in a.family (set by the host's dispatch table), else the
// smallest one whose capacity covers a.max_nb. A family whose capacity is
// below an item's class size flags that grain TMX_ST_TOO_LARGE.
void tmx_launch_blocks(const TmxBlockArgs &a, cudaStream_t stream) {
  if (a.nitems <= 0) {
    return;
  }
  int f = a.family;
  if (f < 0 || f >= TMX_BLOCK_FAMILIES) {
    f = (a.max_nb <= 8)    ? TMX_BLOCKS_WARP_DFMA
        : (a.max_nb <= 16) ? TMX_BLOCKS_WARP_DMMA
        : (a.max_nb <= 32) ? TMX_BLOCKS_CTA32
        : (a.max_nb <= 64) ? TMX_BLOCKS_CTA64
                           : TMX_BLOCKS_CTA;
  }
  switch (f) {
  case TMX_BLOCKS_WARP_DFMA:
    launch_warp_variant<1, 2, TMX_WARP_DFMA_MINB, false>(a, stream);
    return;
  case TMX_BLOCKS_WARP_DMMA:
    launch_warp_variant<1, 1, TMX_WARP_DMMA_MINB, true>(a, stream);
    return;
  case TMX_BLOCKS_CTA32:
    launch_cta32(a, stream);
    return;
  case TMX_BLOCKS_CTA64:
    launch_cta64(a, stream);
    return;
  default: {
    const size_t smem = tmx_block_smem_bytes(a.max_nb, a.chunk_nodes);
    launch_variant<4, 4, 256, 1>(a, smem, stream);
  }
  }
}

// ----------------------------------------------------------- convergence --

// One thread per active slot: m = 0 sums of the latest order in the
// reference's order (TMatrixResource.hpp:743-756) and the convergence test
// (:758-775). Unconverged slots that have orders left go to the next list.
__global__ void k_converge(const int32_t *__restrict__ active, int nactive,
                           const TmxSlot *__restrict__ slots,
                           const cplx *__restrict__ diag, TmxChainState *state,
                           double tolerance, int order, int last_order,
                           int32_t *next_active, int32_t *next_count,
                           int32_t *done_list, int32_t *done_ord,
                           int32_t *done_pos, int32_t *done_count,
                           const int32_t *nact_dev, int base,
                           const int32_t *order_dev) {
  if (order_dev) {
    order = *order_dev;
  }
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nactive || (nact_dev && base + p >= *nact_dev)) {
    return;
  }
  const int g = active[p];
  {
    // speculative orders: a grain whose order became final at an earlier
    // order of the same group is not touched again
    const TmxChainState s0 = state[g];
    if (s0.converged || (s0.status & (TMX_ST_NAN | TMX_ST_NOT_CONVERGED))) {
      return;
    }
  }
  const TmxSlot sl = slots[p];
  const cplx *dg = diag + sl.diag;
  const int N = order;
  double qs = 0., qe = 0.;
  for (int n = 1; n < N + 1; ++n) {
    const double dn1 = 2. * n + 1.;
    const cplx a = dg[n - 1];
    const cplx b = dg[N + n - 1];
    qs += dn1 * (cnorm2(a) + cnorm2(b));
    qe += dn1 * (a.x + b.x);
  }
  TmxChainState st = state[g];
  const double old_qs = st.qsca, old_qe = st.qext;
  st.qsca = qs;
  st.qext = qe;
  st.nmax = N;
  st.ngauss = sl.ngauss;
  if (st.dqs_t == -2.) {
    st.dqs_t = -1.;
    st.dqe_t = -1.;
  } else {
    st.dqs_t = fabs((old_qs - qs) / qs);
    st.dqe_t = fabs((old_qe - qe) / qe);
  }
  if (st.dqs_t > 0.) {
    st.dqs = st.dqs_t;
    st.dqe = st.dqe_t;
    if (st.dqs_t <= tolerance && st.dqe_t <= tolerance) {
      st.converged = 1;
    }
  }
  bool finite = isfinite(qs) && isfinite(qe);
  if (!finite) {
    st.status |= TMX_ST_NAN;
  }
  bool stays = false;
  if (!st.converged && finite) {
    if (order < last_order) {
      const int q = atomicAdd(next_count, 1);
      next_active[q] = g;
      stays = true;
    } else {
      st.status |= TMX_ST_NOT_CONVERGED;
    }
  }
  state[g] = st;
  if (!stays) {
    // the grain's order is final: its blocks may start
    const int q = atomicAdd(done_count, 1);
    done_list[q] = g;
    done_ord[q] = order;
    done_pos[q] = p;
  }
}

void tmx_launch_converge(const int32_t *active, int nactive,
                         const TmxSlot *slots, const double2 *diag,
                         TmxChainState *state, double tolerance, int order,
                         int last_order, int32_t *next_active,
                         int32_t *next_count, int32_t *done_list,
                         int32_t *done_ord, int32_t *done_pos,
                         int32_t *done_count, const int32_t *nact_dev,
                         int base, cudaStream_t stream, const int32_t *order_dev) {
  if (nactive <= 0) {
    return;
  }
  k_converge<<<(nactive + 127) / 128, 128, 0, stream>>>(
      active, nactive, slots, diag, state, tolerance, order, last_order,
      next_active, next_count, done_list, done_ord, done_pos, done_count,
      nact_dev, base, order_dev);
}

// ------------------------------------------------------------- kept tables --

// The node scalars and Bessel tables of a grain's final order are the ones
// its block round needs. Right after the convergence test of a group of
// orders (before the next group overwrites the order loop's table buffers),
// every grain that became final in the group -- done-list entries
// [*next, counters[1]) -- has its tables copied into the batch's arena at a
// reserved offset (in doubles, a multiple of 16), recorded per grain and per
// done-list entry; -1 where the arena is full (the round then recomputes
// them). One CTA per entry, grid-stride; the last CTA to finish moves *next
// to the end of the range.
__global__ void k_keep_tables(TmxKeepArgs K) {
  __shared__ long long s_off;
  __shared__ unsigned s_last;
  if (K.order0_dev) {
    K.order0 = *K.order0_dev;
    K.base[0] = *K.base_dev;
  }
  const int begin = *K.next;
  const int end = K.counters[1];
  for (int q = begin + blockIdx.x; q < end; q += gridDim.x) {
    const int g = K.done_list[q];
    const int s = K.done_ord[q] - K.order0;
    const int p = K.done_pos[q];
    const TmxChainBase b = K.base[s];
    const int64_t tsz = b.tab_stride, nsz = b.nsc_stride;
    const int64_t want = ((tsz + 15) & ~(int64_t)15) + ((nsz + 15) & ~(int64_t)15);
    if (threadIdx.x == 0) {
      const long long off =
          (long long)atomicAdd(K.used, (unsigned long long)want);
      s_off = (off + want <= K.cap) ? off : -1;
    }
    __syncthreads();
    const long long off = s_off;
    if (off >= 0) {
      const double2 *ts = reinterpret_cast<const double2 *>(K.tab + b.tab + p * tsz);
      double2 *td = reinterpret_cast<double2 *>(K.arena + off);
      for (int64_t u = threadIdx.x; u < tsz / 2; u += blockDim.x) {
        td[u] = ts[u];
      }
      const int64_t noff = off + ((tsz + 15) & ~(int64_t)15);
      const double2 *ns = reinterpret_cast<const double2 *>(K.nsc + b.nsc + p * nsz);
      double2 *nd = reinterpret_cast<double2 *>(K.arena + noff);
      for (int64_t u = threadIdx.x; u < nsz / 2; u += blockDim.x) {
        nd[u] = ns[u];
      }
    }
    if (threadIdx.x == 0) {
      K.keep_tab[g] = off;
      K.keep_q[q] = off;
    }
    __syncthreads();
  }
  // the last CTA moves the start of the next range
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    s_last = (atomicAdd(K.ticket, 1u) == gridDim.x - 1) ? 1u : 0u;
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    *K.next = end;
    *K.ticket = 0u;
    __threadfence();
  }
}

void tmx_launch_keep_tables(const TmxKeepArgs &K, int max_entries,
                            cudaStream_t stream) {
  const int blocks = std::max(1, std::min(max_entries, 148 * 4));
  k_keep_tables<<<blocks, 128, 0, stream>>>(K);
}

// ------------------------------------------------------------- Q sums ------

// TMatrixQTask::execute (TMatrixResource.hpp:1136-1210): full Qsca and Qext.
// The reference's quadruple loop over (n1, n2, m1, m2 = m1) visits every
// entry of every m block once, so Qsca = sum_m f_m ||T_m||_F^2 and
// Qext = sum_m f_m sum_n Re(T_m[(0,n),(0,n)] + T_m[(0,n),(1,n)] +
// T_m[(1,n),(0,n)] + T_m[(1,n),(1,n)]), f_0 = 1, f_m = 2. One block per
// grain reads each (contiguous) block coalesced; the reduction order is fixed.
#define QS_THREADS 256
// Qsca and Qext sums of the grains of one block round (TMatrixQTask,
// TMatrixResource.hpp:1136-1210): one CTA per slot, thread t adds the
// entries t, t + 256, ... of every m block in order (|T|^2, and Re T on the
// block diagonals), then a warp tree and the warp partial sums in order.
// Row and column of an entry advance incrementally (no division per entry).
__global__ void __launch_bounds__(QS_THREADS)
    k_qsums(const TmxSlot *__restrict__ slots, int ns,
            const cplx *__restrict__ T, double *q_out,
            const int32_t *__restrict__ range) {
  const int slo = range ? range[0] : 0;
  const int shi = range ? min(range[1], ns) : ns;
  for (int s = slo + blockIdx.x; s < shi; s += gridDim.x) {
  const TmxSlot sl = slots[s];
  const int N = sl.nmax;
  const cplx *Tg = T + sl.tout;
  double qs = 0., qe = 0.;
  for (int m = 0; m <= N && N > 0; ++m) {
    const int nb = (m == 0) ? N : N + 1 - m;
    const int w = 2 * nb;
    const double f = (m > 0) ? 2. : 1.;
    const cplx *B = Tg + block_offset(N, m);
    const int dq = QS_THREADS / w, dr = QS_THREADS % w;
    int row = threadIdx.x / w, col = threadIdx.x % w;
    double bs = 0., be = 0.;
    for (int u = threadIdx.x; u < w * w; u += QS_THREADS) {
      const cplx v = B[u];
      bs += cnorm2(v);
      const int rm = (row >= nb) ? row - nb : row;
      const int cm = (col >= nb) ? col - nb : col;
      if (rm == cm) {
        be += v.x;
      }
      row += dq;
      col += dr;
      if (col >= w) {
        col -= w;
        ++row;
      }
    }
    qs += f * bs;
    qe += f * be;
  }
  __shared__ double red[2][QS_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    qs += __shfl_down_sync(0xffffffffu, qs, o);
    qe += __shfl_down_sync(0xffffffffu, qe, o);
  }
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][warp] = qs;
    red[1][warp] = qe;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0., b = 0.;
    for (int i = 0; i < QS_THREADS / 32; ++i) {
      a += red[0][i];
      b += red[1][i];
    }
    q_out[2 * sl.grain] = a;
    q_out[2 * sl.grain + 1] = b;
  }
  // red is reused by the next slot
  __syncthreads();
  }
}

void tmx_launch_qsums(const TmxSlot *slots, int ns, const cplx *T,
                      double *q_out, cudaStream_t stream, const int32_t *range,
                      int max_ctas) {
  if (ns <= 0) {
    return;
  }
  const int blocks = (max_ctas > 0) ? std::min(ns, max_ctas) : ns;
  k_qsums<<<blocks, QS_THREADS, 0, stream>>>(slots, ns, T, q_out, range);
}

// ------------------------------------------------------------ chain prep --

// Slots and items of one order step: active position p gets the tables at
// p * strides and the four m = 0 classes as items 4p .. 4p + 3.
__global__ void k_chain_prep(const int32_t *__restrict__ active, int nactive,
                             const int32_t *__restrict__ nact_dev, int base,
                             int order, int ngauss, int wig_n, TmxChainBase b,
                             TmxSlot *slots, TmxItem *items) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nactive) {
    return;
  }
  // positions past the list's length on the device (the host launched for
  // an upper bound) get an empty slot: order 0 has no classes and no nodes,
  // so every kernel of the step skips it
  const bool valid = !nact_dev || base + p < *nact_dev;
  TmxSlot s;
  s.grain = valid ? active[p] : 0;
  s.nmax = valid ? order : 0;
  s.ngauss = valid ? ngauss : 0;
  s.wig_n = wig_n;
  s.tab = b.tab + p * b.tab_stride;
  s.nsc = b.nsc + p * b.nsc_stride;
  s.tout = -1;
  s.diag = b.diag + p * b.diag_stride;
  slots[b.slot + p] = s;
  for (int c = 0; c < 4; ++c) {
    TmxItem it;
    it.slot = b.slot + p;
    it.m = 0;
    it.cls = (int16_t)c;
    it.scratch = b.scr + (4 * (int64_t)p + c) * b.scr_stride;
    items[4 * (b.slot + p) + c] = it;
  }
}

void tmx_launch_chain_prep(const int32_t *active, int nactive,
                           const int32_t *nact_dev, int base, int order,
                           int ngauss, int wig_n, const TmxChainBase &b,
                           TmxSlot *slots, TmxItem *items, cudaStream_t stream) {
  if (nactive <= 0) {
    return;
  }
  k_chain_prep<<<(nactive + 127) / 128, 128, 0, stream>>>(
      active, nactive, nact_dev, base, order, ngauss, wig_n, b, slots, items);
}
