// Tangent (forward-mode derivative) kernel of the T-matrix blocks.
//
// For p in {refractive index m (complex derivative), equal-volume radius
// R_V, axis ratio d} and every (grain, m, class) item:
//   dT_c = -(dRgQ_c + T_c dQ_c) Q_c^-1,
// differentiating T_c Q_c = -RgQ_c (the relation T = -RgQ Q^-1 of
// TMatrixResource.hpp:712-730, 1102-1119) and reusing the LU factors of Q_c
// saved by the forward block kernel. The entries of Q and RgQ are
// sum_g sum_t F_t W_t (see tmx_blocks.cu), so dQ = sum [dF W + F dW]: the
// same contraction with the node dimension doubled. All derivatives are
// algebraic in the forward tables; for a spherical Bessel function f of
// argument z and its derivative form df = [z f]'/z (SpecialFunctions.hpp:
// 106-240) the Bessel equation z^2 f'' + 2 z f' + (z^2 - n(n+1)) f = 0 gives
//   d f/dz = df - f/z,   d(df)/dz = n(n+1) f / z^2 - f - df / z.
// Arguments: z = k R_V r(theta), w = m z; dz/dR_V = z/R_V, dw/dm = z,
// dw/dR_V = w/R_V, dz/dd = z (dln r^2/dd)/2; the quadrature weights w r^2
// (and m w r^2 / sin) scale with r^2, so d/dd multiplies them by dln r^2/dd;
// r'/r also depends on d.
#include <algorithm>

#include "tmx_blocks_common.cuh"

extern __shared__ __align__(16) unsigned char tmx_tsmem[];

enum { P_M = 0, P_R = 1, P_D = 2 };

// Tangent chunk: per node 8 slots, slot t (t < 4) pairs F_t with dW_t and
// slot 4 + t pairs dF_t with W_t. For p = m the F side does not depend on
// the parameter and only slots 0..3 are used.
// Threads tid = 0..nth-1 of the caller share the work; rows are stored with
// stride L.NRp, columns with stride ncolp. an_tab[a] = a_n of member a.
__device__ void build_chunk_tangent(const ClassDesc &D, const AsmLayout &L,
                                    int ncolp, int N, int m, int ng, int g0,
                                    int param, double R,
                                    const double *__restrict__ T,
                                    const double *__restrict__ S,
                                    const double *__restrict__ Wg, double k2,
                                    cplx k2mr, cplx *Fs, cplx *Ws, int tid,
                                    int nth, const double *an_tab) {
  const int G = L.G;
  const int slots = 8;
  // ---- A side: F_t (slots 0..3) and dF_t (slots 4..7), (F^j, F^y) pairs
  for (int u = tid; u < G * L.NRp; u += nth) {
    const int gl = u / L.NRp;
    const int pr = u % L.NRp;
    const int g = g0 + gl;
    const int a = padded_member(D, pr);
    cplx f[4], df[4];
    for (int t = 0; t < 4; ++t) {
      f[t] = df[t] = mkc(0., 0.);
    }
    if (a >= 0 && g < ng) {
      int i, n;
      member(D, a, i, n);
      const double *tb = T + ((int64_t)g * N + (n - 1)) * TMX_NQ;
      const double *w = Wg + ((int64_t)g * N + (n - 1)) * 2;
      const double *s = S + (int64_t)g * TMX_NS;
      const double d = w[0], dd = w[1];
      const double an = an_tab[a];
      const double nn = n * (n + 1.);
      const double iz = s[TMX_NS_KRINV];
      const double drr = s[TMX_NS_DRR];
      // h = (j, y) parts handled together
      const double hj = tb[TMX_Q_J], hy = tb[TMX_Q_Y];
      const double dhj = tb[TMX_Q_DJ], dhy = tb[TMX_Q_DY];
      const double q = nn * drr * iz * d;
      f[0] = mkc(an * d * hj, an * d * hy);
      f[1] = mkc(an * dd * hj, an * dd * hy);
      f[2] = mkc(an * d * dhj, an * d * dhy);
      f[3] = mkc(an * (dd * dhj + q * hj), an * (dd * dhy + q * hy));
      if (param != P_M) {
        // d/dz of h, dh and h/z
        const double hpj = dhj - hj * iz, hpy = dhy - hy * iz;
        const double dhpj = nn * hj * iz * iz - hj - dhj * iz;
        const double dhpy = nn * hy * iz * iz - hy - dhy * iz;
        const double hzpj = dhj * iz - 2. * hj * iz * iz;
        const double hzpy = dhy * iz - 2. * hy * iz * iz;
        const double z = s[TMX_NS_KR];
        const double dz = (param == P_R) ? z / R : 0.5 * z * s[TMX_NS_DLNR2_DD];
        const double ddrr = (param == P_D) ? s[TMX_NS_DDRR_DD] : 0.;
        df[0] = mkc(an * d * hpj * dz, an * d * hpy * dz);
        df[1] = mkc(an * dd * hpj * dz, an * dd * hpy * dz);
        df[2] = mkc(an * d * dhpj * dz, an * d * dhpy * dz);
        df[3] = mkc(an * ((dd * dhpj + nn * drr * d * hzpj) * dz +
                          nn * ddrr * d * hj * iz),
                    an * ((dd * dhpy + nn * drr * d * hzpy) * dz +
                          nn * ddrr * d * hy * iz));
      }
    }
    cplx *fp = Fs + (int64_t)(slots * gl) * L.NRp + pr;
    for (int t = 0; t < 4; ++t) {
      fp[t * L.NRp] = f[t];
      fp[(4 + t) * L.NRp] = df[t];
    }
  }
  // ---- B side: dW_t (slots 0..3) and W_t (slots 4..7) for each row group
  for (int u = tid; u < G * ncolp; u += nth) {
    const int gl = u / ncolp;
    const int b = u % ncolp;
    const int g = g0 + gl;
    cplx W[2][4], dW[2][4];
    for (int rg = 0; rg < 2; ++rg) {
      for (int t = 0; t < 4; ++t) {
        W[rg][t] = dW[rg][t] = mkc(0., 0.);
      }
    }
    if (b < D.nb && g < ng) {
      int ib, n;
      member(D, b, ib, n);
      const double *tb = T + ((int64_t)g * N + (n - 1)) * TMX_NQ;
      const cplx jm = mkc(tb[TMX_Q_JM_RE], tb[TMX_Q_JM_IM]);
      const cplx djm = mkc(tb[TMX_Q_DJM_RE], tb[TMX_Q_DJM_IM]);
      const double *w = Wg + ((int64_t)g * N + (n - 1)) * 2;
      const double *s = S + (int64_t)g * TMX_NS;
      const double d = w[0], dd = w[1];
      const double an = an_tab[b];
      const double nn = n * (n + 1.);
      const cplx iw = mkc(s[TMX_NS_KRMRINV_RE], s[TMX_NS_KRMRINV_IM]);
      const double drr = s[TMX_NS_DRR];
      const cplx jw = cmul(jm, iw); // j / w
      const cplx Gv[4] = {
          cscale(djm, an * d),
          cscale(cadd(cscale(djm, dd), cscale(jw, drr * nn * d)), an),
          cscale(jm, an * d), cscale(jm, an * dd)};
      // d/dw of j, dj and j/w
      const cplx iw2 = cmul(iw, iw);
      const cplx jp = csub(djm, jw);
      const cplx djp = csub(csub(cscale(cmul(jm, iw2), nn), jm), cmul(djm, iw));
      const cplx jwp = csub(cmul(djm, iw), cscale(cmul(jm, iw2), 2.));
      // dw/dp
      const cplx wv = mkc(s[TMX_NS_KRMR_RE], s[TMX_NS_KRMR_IM]);
      cplx dw;
      if (param == P_M) {
        dw = mkc(s[TMX_NS_KR], 0.);
      } else if (param == P_R) {
        dw = cscale(wv, 1. / R);
      } else {
        dw = cscale(wv, 0.5 * s[TMX_NS_DLNR2_DD]);
      }
      const double ddrr = (param == P_D) ? s[TMX_NS_DDRR_DD] : 0.;
      const cplx dGv[4] = {
          cmul(cscale(djp, an * d), dw),
          cadd(cmul(cscale(cadd(cscale(djp, dd), cscale(jwp, drr * nn * d)), an), dw),
               cscale(jw, an * nn * d * ddrr)),
          cmul(cscale(jp, an * d), dw), cmul(cscale(jp, an * dd), dw)};
      const double wr2 = s[TMX_NS_W] * s[TMX_NS_R2];
      const double mu = (double)(m * m) * s[TMX_NS_SIN2INV];
      const double beta = s[TMX_NS_SININV] * m * wr2;
      // d(weight)/dp / weight: r^2 scales the weights when d changes
      const double lw = (param == P_D) ? s[TMX_NS_DLNR2_DD] : 0.;
      const cplx k2c = mkc(k2, 0.);
      const cplx dk2mr = (param == P_M) ? k2c : mkc(0., 0.);
      for (int rg = 0; rg < L.ngroups; ++rg) {
        const int ia = (rg == 0) ? D.iA : D.iB;
        if (ia == ib) {
          const cplx chi = (ia == 0) ? k2mr : k2c;
          const cplx clo = (ia == 0) ? mkc(-k2, 0.) : mkc(-k2mr.x, -k2mr.y);
          const cplx dchi = (ia == 0) ? dk2mr : mkc(0., 0.);
          const cplx dclo = (ia == 0) ? mkc(0., 0.) : mkc(-dk2mr.x, -dk2mr.y);
          const double wts[4] = {wr2 * mu, wr2, wr2 * mu, wr2};
          for (int t = 0; t < 4; ++t) {
            const cplx c = (t < 2) ? chi : clo;
            const cplx dc = (t < 2) ? dchi : dclo;
            W[rg][t] = cmul(c, cscale(Gv[t], wts[t]));
            // d(c w G) = dc w G + c (lw w) G + c w dG
            dW[rg][t] = cadd(cmul(dc, cscale(Gv[t], wts[t])),
                             cmul(c, cadd(cscale(Gv[t], wts[t] * lw),
                                          cscale(dGv[t], wts[t]))));
          }
        } else {
          const cplx c1 = (ia == 0) ? k2mr : k2c;
          const cplx c2 = (ia == 0) ? k2c : k2mr;
          const cplx dc1 = (ia == 0) ? dk2mr : mkc(0., 0.);
          const cplx dc2 = (ia == 0) ? mkc(0., 0.) : dk2mr;
          const int gi[4] = {3, 2, 1, 0};
          for (int t = 0; t < 4; ++t) {
            const cplx c = (t < 2) ? c1 : c2;
            const cplx dc = (t < 2) ? dc1 : dc2;
            const cplx ic = mkc(-c.y * beta, c.x * beta);    // i c beta
            const cplx idc = mkc(-dc.y * beta, dc.x * beta); // i dc beta
            const cplx Gt = Gv[gi[t]];
            W[rg][t] = cmul(ic, Gt);
            dW[rg][t] = cadd(cmul(idc, Gt),
                             cmul(ic, cadd(cscale(Gt, lw), dGv[gi[t]])));
          }
        }
      }
    }
    for (int rg = 0; rg < L.ngroups; ++rg) {
      cplx *wp = Ws + ((int64_t)rg * slots * G + slots * gl) * ncolp + b;
      for (int t = 0; t < 4; ++t) {
        wp[t * ncolp] = dW[rg][t];
        wp[(4 + t) * ncolp] = W[rg][t];
      }
    }
  }
}

// One block per (item, parameter).
template <int TR, int TC, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_tangent(TmxTangentArgs A, size_t smem_bytes) {
  const int it = blockIdx.x;
  const int param = blockIdx.y;
  if (it >= A.nitems || param >= A.nparams) {
    return;
  }
  const TmxItem item = A.items[it];
  const TmxSlot sl = A.slots[item.slot];
  const TmxGrain Gr = A.grains[sl.grain];
  const int N = sl.nmax;
  const int ng = sl.ngauss;
  const int m = item.m;
  const ClassDesc D = describe<TR>(N, m, item.cls);
  const int nb = D.nb;
  // (shared memory is sized for classes of at most max_nb members)
  if (nb <= 0 || nb > TMX_MAX_NB || nb > A.max_nb) {
    return;
  }
  const double *T = A.tab + sl.tab;
  const double *S = A.nsc + sl.nsc;
  const double *Wg = A.wig + A.wig_off[sl.wig_n] + (int64_t)m * ng * N * 2;
  const double k2 = Gr.k * Gr.k;
  const cplx k2mr = mkc(Gr.mr * k2, Gr.mi * k2);
  cplx *dQ = A.scratch + param * A.scratch_stride + item.scratch;
  cplx *dR = dQ + (int64_t)nb * nb;
  __shared__ double an_tab[TMX_MAX_NB];
  for (int a = threadIdx.x; a < nb; a += blockDim.x) {
    int ia, na;
    member(D, a, ia, na);
    an_tab[a] = a_n(na);
  }

  // ---------------------------------------------------- tangent assembly
  AsmLayout L;
  L.G = A.chunk_nodes;
  L.NRp = D.NRp;
  L.CT = (nb + TC - 1) / TC;
  L.ncol = L.CT * TC;
  L.ngroups = (D.R1 > 0 && m > 0) ? 2 : 1;
  const int RT = D.NRp / TR;
  cplx *Fs = reinterpret_cast<cplx *>(tmx_tsmem);
  cplx *Ws = Fs + (int64_t)8 * L.G * L.NRp;
  const int ntiles = RT * L.CT;
  const int tstep = (m == 0) ? 2 : 1;
  const int t0 = (m == 0) ? 1 : 0;
  const int per_node = (param == P_M) ? 4 : 8;
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
      build_chunk_tangent(D, L, L.CT * TC, N, m, ng, g0, param, Gr.r_ev, T, S,
                          Wg, k2, k2mr, Fs, Ws, threadIdx.x, blockDim.x, an_tab);
      __syncthreads();
      if (active) {
        const int gmax = min(L.G, ng - g0);
        for (int gl = 0; gl < gmax; ++gl) {
          for (int ts = t0; ts < per_node; ts += tstep) {
            const int kk = 8 * gl + ts;
            const cplx *fr = Fs + (int64_t)kk * L.NRp + rt * TR;
            const cplx *wr = Ws + ((int64_t)rg * 8 * L.G + kk) * L.ncol + ct;
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
          dQ[(int64_t)a * nb + b] =
              mkc(aj[r][c][0] - ay[r][c][1], aj[r][c][1] + ay[r][c][0]);
          dR[(int64_t)a * nb + b] = mkc(aj[r][c][0], aj[r][c][1]);
        }
      }
    }
  }
  __syncthreads();

  // ---------------------------------------- solve with the saved factors
  if constexpr (NT == 128) {
    // classes of up to 32 members: T_c and the factors in shared memory,
    // B = dRgQ + T_c dQ by all threads, then the register solve with four
    // lanes per row (row tid / 4)
    constexpr int LF = 33;
    if (nb <= 32) {
      cplx *Am = reinterpret_cast<cplx *>(tmx_tsmem);
      cplx *Tc = Am + 32 * LF;
      cplx *Xs = Tc + 32 * LF;
      cplx *uinv = Xs + 32 * LF;
      int *perm = reinterpret_cast<int *>(uinv + 32);
      const cplx *Ls = A.lu + item.scratch;
      const int *ps = reinterpret_cast<const int *>(Ls + (int64_t)nb * nb);
      const cplx *Tb = A.T + sl.tout + block_offset(N, m);
      const int w2 = 2 * D.nbb;
      for (int u = threadIdx.x; u < nb * nb; u += NT) {
        const int a = u / nb;
        const int k = u - a * nb;
        Am[a * LF + k] = Ls[u];
        int ia, na, ik, nk;
        member(D, a, ia, na);
        member(D, k, ik, nk);
        Tc[a * LF + k] = Tb[(int64_t)(ia * D.nbb + (na - D.nmin)) * w2 + ik * D.nbb +
                            (nk - D.nmin)];
      }
      for (int j = threadIdx.x; j < nb; j += NT) {
        perm[j] = ps[j];
        uinv[j] = cinv_lu(Ls[(int64_t)j * nb + j]);
      }
      __syncthreads();
      for (int u = threadIdx.x; u < nb * nb; u += NT) {
        const int a = u / nb;
        const int b = u - a * nb;
        cplx acc = dR[u];
        for (int k = 0; k < nb; ++k) {
          acc = cadd(acc, cmul(Tc[a * LF + k], dQ[(int64_t)k * nb + b]));
        }
        Xs[a * LF + b] = acc;
      }
      __syncthreads();
      solve_rows<32, 4>(Xs, Am, LF, uinv, nb, threadIdx.x >> 2, threadIdx.x & 3);
      __syncthreads();
      cplx *dTb = A.dT + param * A.dT_stride + sl.tout + block_offset(N, m);
      for (int u = threadIdx.x; u < nb * nb; u += NT) {
        const int a = u / nb;
        const int b = u - a * nb;
        int ia, na, ib, nbn;
        member(D, a, ia, na);
        member(D, b, ib, nbn);
        dTb[(int64_t)(ia * D.nbb + (na - D.nmin)) * w2 + ib * D.nbb + (nbn - D.nmin)] =
            Xs[a * LF + perm[b]];
      }
      return;
    }
  }
  const int lda = nb | 1;
  cplx *Am = reinterpret_cast<cplx *>(tmx_tsmem);
  cplx *uinv = Am + (int64_t)nb * lda;
  int *perm = reinterpret_cast<int *>(uinv + nb);
  size_t used = ((size_t)nb * lda + nb) * sizeof(cplx) + nb * sizeof(int);
  used = (used + 15) & ~(size_t)15;
  cplx *X = reinterpret_cast<cplx *>(tmx_tsmem + used);
  int Rchunk = (int)((smem_bytes - used) / (sizeof(cplx) * lda));
  if (Rchunk > nb) {
    Rchunk = nb;
  }
  const cplx *Ls = A.lu + item.scratch;
  const int *ps = reinterpret_cast<const int *>(Ls + (int64_t)nb * nb);
  for (int u = threadIdx.x; u < nb * nb; u += blockDim.x) {
    Am[(u / nb) * lda + (u % nb)] = Ls[u];
  }
  for (int j = threadIdx.x; j < nb; j += blockDim.x) {
    perm[j] = ps[j];
    uinv[j] = cinv(Ls[(int64_t)j * nb + j]);
  }
  __syncthreads();
  const cplx *Tb = A.T + sl.tout + block_offset(N, m);
  cplx *dTb = A.dT + param * A.dT_stride + sl.tout + block_offset(N, m);
  const int w2 = 2 * D.nbb;
  for (int r0 = 0; r0 < nb; r0 += Rchunk) {
    const int R = min(Rchunk, nb - r0);
    // X = -(dRgQ + T_c dQ) for rows r0 .. r0 + R
    for (int u = threadIdx.x; u < R * nb; u += blockDim.x) {
      const int r = u / nb;
      const int b = u % nb;
      const int a = r0 + r;
      int ia, na;
      member(D, a, ia, na);
      const cplx *trow = Tb + (int64_t)(ia * D.nbb + (na - D.nmin)) * w2;
      cplx acc = dR[(int64_t)a * nb + b];
      for (int k = 0; k < nb; ++k) {
        int ik, nk;
        member(D, k, ik, nk);
        acc = cadd(acc, cmul(trow[ik * D.nbb + (nk - D.nmin)], dQ[(int64_t)k * nb + b]));
      }
      X[r * lda + b] = mkc(-acc.x, -acc.y);
    }
    __syncthreads();
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
    for (int j = nb - 1; j >= 1; --j) {
      for (int u = threadIdx.x; u < R * j; u += blockDim.x) {
        const int r = u / j;
        const int k = u % j;
        X[r * lda + k] = csub(X[r * lda + k], cmul(X[r * lda + j], Am[j * lda + k]));
      }
      __syncthreads();
    }
    for (int u = threadIdx.x; u < R * nb; u += blockDim.x) {
      const int r = u / nb;
      const int b = u % nb;
      const int a = r0 + r;
      int ia, na, ib, nbn;
      member(D, a, ia, na);
      member(D, b, ib, nbn);
      dTb[(int64_t)(ia * D.nbb + (na - D.nmin)) * w2 + ib * D.nbb + (nbn - D.nmin)] =
          X[r * lda + perm[b]];
    }
    __syncthreads();
  }
}

// ------------------------------------------------- warp-per-item variant --
//
// (item, parameter) pairs of classes with at most 16 members: one warp each,
// four per CTA, synchronised by __syncwarp only (as the forward warp kernel).
// Assembly: lane (rt, ct) accumulates rows rt * TR.. and columns ct, ct + 4,
// .. over chunks of TMX_TWG nodes. Solve: lane r forms row r of
// X = -(dRgQ + T_c dQ) and runs both triangular solves with the saved
// factors on it.

#define TMX_TWG 2 // quadrature nodes per warp chunk

template <int NBM>
__host__ __device__ constexpr int tangent_warp_elems() {
  // chunk buffers F[WG][8][NBM] + W[2][WG][8][NBM], or in the solve phase
  // dQ, X, LU, T_c ([NBM][NBM + 1] each), 1/U_jj and the gather index
  return (24 * TMX_TWG * NBM > 4 * NBM * (NBM + 1) + 2 * NBM)
             ? 24 * TMX_TWG * NBM
             : 4 * NBM * (NBM + 1) + 2 * NBM;
}

template <int TR, int TC, int MINB>
__global__ void __launch_bounds__(128, MINB)
    k_tangent_warp(TmxTangentArgs A) {
  constexpr int NBM = (8 * TR > 4 * TC) ? 8 * TR : 4 * TC;
  constexpr int LD = NBM + 1;
  extern __shared__ __align__(16) unsigned char tmx_twsmem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  cplx *base = reinterpret_cast<cplx *>(tmx_twsmem) + wib * tangent_warp_elems<NBM>();
  cplx *Fs = base;                       // [WG][8][NBM]
  cplx *Ws = Fs + 8 * TMX_TWG * NBM;     // [2][WG][8][NBM]
  cplx *dQm = base;                      // [NBM][LD]  (after the assembly)
  cplx *Xm = dQm + NBM * LD;             // [NBM][LD]
  cplx *LUm = Xm + NBM * LD;             // [NBM][LD]
  cplx *Tcm = LUm + NBM * LD;            // [NBM][LD]
  cplx *uinv = Tcm + NBM * LD;           // [NBM]
  int *perm = reinterpret_cast<int *>(uinv + NBM);
  __shared__ double an_w[4][NBM];
  double *an_tab = an_w[wib];
  const int rt = lane >> 2;
  const int ct = lane & 3;
  const int64_t nwork = (int64_t)A.nitems * A.nparams;
  for (int64_t w = (int64_t)blockIdx.x * 4 + wib; w < nwork;
       w += (int64_t)gridDim.x * 4) {
    const int it = (int)(w / A.nparams);
    const int param = (int)(w % A.nparams);
    const TmxItem item = A.items[it];
    const TmxSlot sl = A.slots[item.slot];
    const TmxGrain Gr = A.grains[sl.grain];
    const int N = sl.nmax;
    const int ng = sl.ngauss;
    const int m = item.m;
    const ClassDesc D = describe<TR>(N, m, item.cls);
    const int nb = D.nb;
    if (nb <= 0 || nb > NBM || D.NRp > NBM) {
      continue;
    }
    const double *T = A.tab + sl.tab;
    const double *S = A.nsc + sl.nsc;
    const double *Wg = A.wig + A.wig_off[sl.wig_n] + (int64_t)m * ng * N * 2;
    const double k2 = Gr.k * Gr.k;
    const cplx k2mr = mkc(Gr.mr * k2, Gr.mi * k2);
    AsmLayout L;
    L.G = TMX_TWG;
    L.NRp = NBM;
    L.CT = 0;
    L.ncol = NBM;
    L.ngroups = (D.R1 > 0 && m > 0) ? 2 : 1;
    const int tstep = (m == 0) ? 2 : 1;
    const int t0 = (m == 0) ? 1 : 0;
    const int per_node = (param == P_M) ? 4 : 8;
    const int rgl = (rt * TR < D.R0p) ? 0 : 1;
    __syncwarp();
    if (lane < nb) {
      int ia, na;
      member(D, lane, ia, na);
      an_tab[lane] = a_n(na);
    }

    // -------------------------------------------------- tangent assembly
    double aj[TR][TC][2], ay[TR][TC][2];
#pragma unroll
    for (int r = 0; r < TR; ++r) {
#pragma unroll
      for (int c = 0; c < TC; ++c) {
        aj[r][c][0] = aj[r][c][1] = ay[r][c][0] = ay[r][c][1] = 0.;
      }
    }
    for (int g0 = 0; g0 < ng; g0 += TMX_TWG) {
      __syncwarp();
      build_chunk_tangent(D, L, NBM, N, m, ng, g0, param, Gr.r_ev, T, S, Wg, k2,
                          k2mr, Fs, Ws, lane, 32, an_tab);
      __syncwarp();
      const int gmax = min(TMX_TWG, ng - g0);
      for (int gl = 0; gl < gmax; ++gl) {
        for (int ts = t0; ts < per_node; ts += tstep) {
          const int kk = 8 * gl + ts;
          const cplx *fr = Fs + kk * NBM + rt * TR;
          const cplx *wr = Ws + (rgl * 8 * TMX_TWG + kk) * NBM + ct;
          cplx wv[TC];
#pragma unroll
          for (int c = 0; c < TC; ++c) {
            wv[c] = wr[4 * c];
          }
#pragma unroll
          for (int r = 0; r < TR; ++r) {
            const cplx f = fr[r];
#pragma unroll
            for (int c = 0; c < TC; ++c) {
              aj[r][c][0] = fma(f.x, wv[c].x, aj[r][c][0]);
              aj[r][c][1] = fma(f.x, wv[c].y, aj[r][c][1]);
              ay[r][c][0] = fma(f.y, wv[c].x, ay[r][c][0]);
              ay[r][c][1] = fma(f.y, wv[c].y, ay[r][c][1]);
            }
          }
        }
      }
    }
    __syncwarp();
    // dQ = dG^j + i dG^y into dQm, dRgQ = dG^j into Xm
#pragma unroll
    for (int r = 0; r < TR; ++r) {
      const int a = padded_member(D, rt * TR + r);
#pragma unroll
      for (int c = 0; c < TC; ++c) {
        const int b = ct + 4 * c;
        if (a >= 0 && b < nb) {
          dQm[a * LD + b] = mkc(aj[r][c][0] - ay[r][c][1], aj[r][c][1] + ay[r][c][0]);
          Xm[a * LD + b] = mkc(aj[r][c][0], aj[r][c][1]);
        }
      }
    }
    // saved factors, gather index and T_c (class order) of the forward solve
    const cplx *Ls = A.lu + item.scratch;
    const int *ps = reinterpret_cast<const int *>(Ls + (int64_t)nb * nb);
    const cplx *Tb = A.T + sl.tout + block_offset(N, m);
    const int w2 = 2 * D.nbb;
    for (int u = lane; u < nb * nb; u += 32) {
      const int a = u / nb;
      const int k = u - a * nb;
      LUm[a * LD + k] = Ls[u];
      int ia, na, ik, nk;
      member(D, a, ia, na);
      member(D, k, ik, nk);
      Tcm[a * LD + k] = Tb[(int64_t)(ia * D.nbb + (na - D.nmin)) * w2 + ik * D.nbb +
                           (nk - D.nmin)];
    }
    for (int j = lane; j < nb; j += 32) {
      perm[j] = ps[j];
      uinv[j] = cinv_lu(Ls[(int64_t)j * nb + j]);
    }
    __syncwarp();
    // ------------------- B = dRgQ + T_c dQ; the solve takes X = -B and
    // solves X U = -B, then Y L = X
    for (int u = lane; u < nb * nb; u += 32) {
      const int a = u / nb;
      const int b = u - a * nb;
      cplx acc = Xm[a * LD + b];
      for (int k = 0; k < nb; ++k) {
        acc = cadd(acc, cmul(Tcm[a * LD + k], dQm[k * LD + b]));
      }
      Xm[a * LD + b] = acc;
    }
    __syncwarp();
    solve_rows<NBM, 32 / NBM>(Xm, LUm, LD, uinv, nb, lane / (32 / NBM),
                              lane % (32 / NBM));
    __syncwarp();
    cplx *dTb = A.dT + param * A.dT_stride + sl.tout + block_offset(N, m);
    for (int u = lane; u < nb * nb; u += 32) {
      const int a = u / nb;
      const int b = u - a * nb;
      int ia, na, ib, nbn;
      member(D, a, ia, na);
      member(D, b, ib, nbn);
      dTb[(int64_t)(ia * D.nbb + (na - D.nmin)) * w2 + ib * D.nbb + (nbn - D.nmin)] =
          Xm[a * LD + perm[b]];
    }
    __syncwarp();
  }
}

template <int TR, int TC, int MINB>
static void launch_tangent_warp(const TmxTangentArgs &a, cudaStream_t stream) {
  constexpr int NBM = (8 * TR > 4 * TC) ? 8 * TR : 4 * TC;
  const size_t smem = (size_t)4 * tangent_warp_elems<NBM>() * sizeof(cplx);
  cudaFuncSetAttribute(k_tangent_warp<TR, TC, MINB>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  // one (item, parameter) per warp: CTAs retire quickly, so that the
  // launches of the other size buckets running beside this one get SMs
  const int64_t work = (int64_t)a.nitems * a.nparams;
  const int blocks = (int)std::max<int64_t>(1, (work + 3) / 4);
  k_tangent_warp<TR, TC, MINB><<<blocks, 128, smem, stream>>>(a);
}

size_t tmx_tangent_smem_bytes(int max_nb, int chunk_nodes) {
  const int nrp = (max_nb + 3) / 4 * 4 + 4;
  const int ncol = (max_nb + 3) / 4 * 4;
  const size_t asm_bytes =
      ((size_t)8 * chunk_nodes * nrp + (size_t)2 * 8 * chunk_nodes * ncol) *
      sizeof(cplx);
  const int lda = max_nb | 1;
  size_t lu = ((size_t)max_nb * lda + max_nb) * sizeof(cplx) + max_nb * sizeof(int);
  lu = (lu + 15) & ~(size_t)15;
  const int rows = max_nb < 8 ? max_nb : 8;
  size_t lu_total = lu + (size_t)rows * lda * sizeof(cplx);
  const size_t full = lu + (size_t)max_nb * lda * sizeof(cplx);
  if (full <= 200 * 1024) {
    lu_total = full;
  }
  if (max_nb <= 32) {
    // solve of the 128-thread kernel: factors, T_c and B (32 x 33 each),
    // 1/U_jj and the gather index
    const size_t small = (size_t)(3 * 32 * 33 + 32) * sizeof(cplx) + 32 * sizeof(int);
    lu_total = std::max(lu_total, small);
  }
  return asm_bytes > lu_total ? asm_bytes : lu_total;
}

template <int TR, int TC, int NT, int MINB>
static void launch_tangent(const TmxTangentArgs &a, size_t smem,
                           cudaStream_t stream) {
  static int attr_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    // the block limit (227 KiB) covers the kernel's static shared memory too
    cudaFuncAttributes fa;
    cudaFuncGetAttributes(&fa, k_tangent<TR, TC, NT, MINB>);
    cudaFuncSetAttribute(k_tangent<TR, TC, NT, MINB>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(227 * 1024 - fa.sharedSizeBytes));
    attr_dev = dev;
  }
  dim3 grid(a.nitems, a.nparams);
  k_tangent<TR, TC, NT, MINB><<<grid, NT, smem, stream>>>(a, smem);
}

void tmx_launch_tangents(const TmxTangentArgs &a, cudaStream_t stream) {
  if (a.nitems <= 0 || a.nparams <= 0) {
    return;
  }
  if (a.max_nb <= 8) {
    launch_tangent_warp<1, 2, 3>(a, stream);
    return;
  }
  if (a.max_nb <= 16) {
    launch_tangent_warp<2, 4, 2>(a, stream);
    return;
  }
  const size_t smem = tmx_tangent_smem_bytes(a.max_nb, a.chunk_nodes);
  if (a.max_nb <= 32) {
    launch_tangent<2, 4, 128, 3>(a, smem, stream);
  } else {
    launch_tangent<4, 4, 256, 1>(a, smem, stream);
  }
}
