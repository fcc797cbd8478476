// Parity-class descriptors and helpers shared by the block kernels.
#pragma once

#include "tmx_common.cuh"
#include "tmx_kernels.h"

// Thread tiles: every thread of the assembly owns TR rows x TC columns of the
// class matrix (columns strided by the column-tile count for conflict-free
// shared-memory reads). Small classes use small tiles and small blocks so
// that many blocks fit on an SM.

struct ClassDesc {
  int nb;       // class size
  int R0, R1;   // rows of group 0 / group 1
  int R0p, NRp; // padded group-0 rows, padded total rows
  int iA, iB;   // block index i of group 0 / group 1
  int nA0, nB0; // first n of each group (n advances by 2)
  int nbb;      // size nb of the full block (2 nbb x 2 nbb)
  int nmin;     // smallest n in the block
};

template <int TR>
__device__ __forceinline__ ClassDesc describe(int N, int m, int cls) {
  ClassDesc D;
  if (m == 0) {
    D.iA = cls >> 1;
    D.iB = D.iA;
    D.nA0 = (cls & 1) ? 1 : 2;
    D.R0 = (N >= D.nA0) ? (N - D.nA0) / 2 + 1 : 0;
    D.nB0 = 0;
    D.R1 = 0;
    D.nbb = N;
    D.nmin = 1;
  } else {
    D.iA = 0;
    D.iB = 1;
    D.nA0 = ((m & 1) == cls) ? m : m + 1;
    D.R0 = (N >= D.nA0) ? (N - D.nA0) / 2 + 1 : 0;
    D.nB0 = ((m & 1) == (cls ^ 1)) ? m : m + 1;
    D.R1 = (N >= D.nB0) ? (N - D.nB0) / 2 + 1 : 0;
    D.nbb = N + 1 - m;
    D.nmin = m;
  }
  D.nb = D.R0 + D.R1;
  D.R0p = (D.R0 + TR - 1) / TR * TR;
  D.NRp = D.R0p + (D.R1 + TR - 1) / TR * TR;
  return D;
}

__device__ __forceinline__ void member(const ClassDesc &D, int a, int &i,
                                       int &n) {
  if (a < D.R0) {
    i = D.iA;
    n = D.nA0 + 2 * a;
  } else {
    i = D.iB;
    n = D.nB0 + 2 * (a - D.R0);
  }
}

// padded row -> member (or -1 for padding)
__device__ __forceinline__ int padded_member(const ClassDesc &D, int pr) {
  if (pr < D.R0p) {
    return (pr < D.R0) ? pr : -1;
  }
  const int a = D.R0 + (pr - D.R0p);
  return (pr - D.R0p < D.R1) ? a : -1;
}

// complex offset of block m in a T-matrix of order N (reference layout)
__device__ __host__ __forceinline__ int64_t block_offset(int N, int m) {
  if (m == 0) {
    return 0;
  }
  const int64_t a = N, b = N + 1 - m;
  const int64_t sa = a * (a + 1) * (2 * a + 1) / 6;
  const int64_t sb = b * (b + 1) * (2 * b + 1) / 6;
  return 4 * (a * a + sa - sb);
}

__device__ __forceinline__ double a_n(int n) {
  // a_n = sqrt((2n + 1) / (n (n + 1))) (NBasedResources.hpp:115-137)
  return sqrt((2. * n + 1.) / ((n + 1.) * n));
}

// Shared-memory layout of the assembly phase for a chunk of G nodes:
//   F[kk][pr]   double2 (F^j, F^y),  kk = 4 * gl + t,   pr < NRp
//   W[rg][kk][b] double2 (complex),  rg = row group,    b < CT * TC
struct AsmLayout {
  int G, NRp, CT, ncol, ngroups;
  size_t f_elems, w_elems;
};


// hypot without the libm scaling path; the magnitudes here are far from
// overflow/underflow
__device__ __forceinline__ double cabs_dev(cplx a) { return hypot(a.x, a.y); }

// 1 / z for the LU pivots and diagonals: conj(z) / |z|^2 on z scaled by the
// power of two 2^-e, e the exponent of max(|Re z|, |Im z|) (exact scaling,
// so |z|^2 lies in [1, 8) and neither overflows nor underflows); one real
// division where Smith's quotient takes two in sequence.
__device__ __forceinline__ cplx cinv_lu(cplx z) {
  const double mx = fmax(fabs(z.x), fabs(z.y));
  const int e = ((__double2hiint(mx) >> 20) & 0x7ff) - 1023;
  const int be = min(max(1023 - e, 1), 2046);
  const double s = __hiloint2double(be << 20, 0); // 2^-e
  const double a = z.x * s, b = z.y * s;
  const double r = 1. / (a * a + b * b);
  return mkc((a * r) * s, (-b * r) * s);
}

// Solve X U = -B, then Y L = X (L unit lower) for row `row` of B (in Rm,
// overwritten by Y) with the factors in Qm and 1/U_jj in uinv; C lanes per
// row (a group of C consecutive lanes), lane c of the group on columns
// c + C t.
template <int NBM, int C>
__device__ __forceinline__ void solve_rows(cplx *Rm, const cplx *Qm, int LD,
                                           const cplx *uinv, int nb, int row,
                                           int c) {
  constexpr int NT = NBM / C;
  const bool act = row < nb;
  cplx x[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    const int k = c + C * t;
    const cplx v = (act && k < nb) ? Rm[row * LD + k] : mkc(0., 0.);
    x[t] = mkc(-v.x, -v.y);
  }
  // Z U = X (forward over columns)
#pragma unroll
  for (int j = 0; j < NBM; ++j) {
    if (j >= nb) {
      break;
    }
    cplx xj = mkc(0., 0.);
    if (c == j % C) {
      xj = cmul(x[j / C], uinv[j]);
      x[j / C] = xj;
    }
    xj.x = __shfl_sync(0xffffffffu, xj.x, j % C, C);
    xj.y = __shfl_sync(0xffffffffu, xj.y, j % C, C);
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int k = c + C * t;
      if (k > j && k < nb) {
        x[t] = csub(x[t], cmul(xj, Qm[j * LD + k]));
      }
    }
  }
  // Y L = Z (backward over columns)
#pragma unroll
  for (int j = NBM - 1; j >= 1; --j) {
    if (j < nb) {
      cplx xj;
      xj.x = __shfl_sync(0xffffffffu, x[j / C].x, j % C, C);
      xj.y = __shfl_sync(0xffffffffu, x[j / C].y, j % C, C);
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const int k = c + C * t;
        if (k < j) {
          x[t] = csub(x[t], cmul(xj, Qm[j * LD + k]));
        }
      }
    }
  }
  if (act) {
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int k = c + C * t;
      if (k < nb) {
        Rm[row * LD + k] = x[t];
      }
    }
  }
}
