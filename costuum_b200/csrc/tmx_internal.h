// Internal declarations shared by the host driver and the CUDA kernels.
#pragma once

#include <stdint.h>

// Per-grain constants, computed on the host with the C library so that they
// carry the same bits as the reference's InteractionVariables
// (src/InteractionResource.hpp:50-132) and get_r_dr_spheroid (cbrt(d)).
struct TmxGrain {
  double r_ev;       // equal-volume radius R_V (m)
  double k;          // wavenumber 2 pi / lambda (1/m)
  double mr, mi;     // refractive index
  double axis_ratio; // d = a / b
  double cbrt_d;     // cbrt(d)
};

// Layout of the per-grain tables at one (nmax, ngauss):
//   node scalars  nsc[g * TMX_NS + s], g < ngauss (lower-half nodes)
//   Bessel table  tab[(g * nmax + (n - 1)) * TMX_NQ + q]
enum {
  TMX_NS_KRINV = 0,
  TMX_NS_KRMRINV_RE,
  TMX_NS_KRMRINV_IM,
  TMX_NS_R2,
  TMX_NS_DRR,
  TMX_NS_W,
  TMX_NS_COS,
  TMX_NS_SININV,
  TMX_NS_SIN2INV,
  TMX_NS_KR,        // k r R_V
  TMX_NS_KRMR_RE,   // m k r R_V
  TMX_NS_KRMR_IM,
  TMX_NS_DLNR2_DD,  // d ln(r^2) / d(axis ratio)
  TMX_NS_DDRR_DD,   // d (r'/r) / d(axis ratio)
  TMX_NS_PAD,       // two pads: a node's row is 128 bytes, so rows are
  TMX_NS_PAD2,      // 16-byte aligned for asynchronous copies
  TMX_NS
};
static_assert(TMX_NS == 16, "node-scalar rows of 16 doubles");
enum {
  TMX_Q_J = 0, // j_n(kr)
  TMX_Q_DJ,    // [kr j_n(kr)]' / kr
  TMX_Q_Y,     // y_n(kr)
  TMX_Q_DY,    // [kr y_n(kr)]' / kr
  TMX_Q_JM_RE, // j_n(m kr)
  TMX_Q_JM_IM,
  TMX_Q_DJM_RE, // [m kr j_n(m kr)]' / (m kr)
  TMX_Q_DJM_IM,
  TMX_NQ
};

// One unit of block work: (grain, m, parity class). Classes: for m >= 1,
// cls in {0, 1} collects the rows (i, n) with (i + n) % 2 == cls; for m = 0,
// cls in {0..3} is (i = cls >> 1, n odd if cls & 1 else even).
struct TmxItem {
  int32_t slot;    // index into the per-slot arrays (grain state/tables)
  int16_t m;
  int16_t cls;
  int64_t scratch; // offset (complex elements) of this item's Q/RgQ scratch
};

// Per-slot descriptor for the block kernel.
struct TmxSlot {
  int32_t grain;  // grain index
  int32_t nmax;
  int32_t ngauss;
  int32_t wig_n;  // index of the Wigner table set for this nmax
  int64_t tab;    // offset of the Bessel table (doubles)
  int64_t nsc;    // offset of the node scalars (doubles)
  int64_t tout;   // offset of the T-matrix (complex elements); -1: chain mode
  int64_t diag;   // offset of the chain-mode diagonal buffer (complex)
};

// status bits (per grain)
enum {
  TMX_ST_OK = 0,
  TMX_ST_NOT_CONVERGED = 1,   // chain reached maximum_order - 1
  TMX_ST_SINGULAR = 2,        // zero pivot in a Q block
  TMX_ST_NAN = 4,             // NaN/Inf in a result
  TMX_ST_BAD_INPUT = 8,       // invalid grain parameters
  TMX_ST_TOO_LARGE = 16,      // block larger than the kernel supports
};

#define TMX_MAX_NB 128 // largest class size handled on chip

// block-kernel families (values of tmx_block_family in tmx.h)
enum {
  TMX_BLOCKS_WARP_DFMA = 0, // warp per item, DFMA register tiles, nb <= 8
  TMX_BLOCKS_WARP_DMMA = 1, // warp per item, DMMA m8n8k4 tiles, nb <= 16
  TMX_BLOCKS_CTA32 = 2,     // four warps per item, nb <= 32
  TMX_BLOCKS_CTA64 = 3,     // eight warps per item, nb <= 64
  TMX_BLOCKS_CTA = 4,       // 256 threads per item, 4x4 tiles, nb <= 128
  TMX_BLOCK_FAMILIES = 5
};

// orders above max(nmax, |z|) at which the Bessel ratio recurrence starts
// when no fixed start is requested
#define TMX_BESSEL_MARGIN 48
