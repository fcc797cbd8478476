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
