// T-matrix at a fixed (nmax, ngauss) without any device allocation.
//
// Some callers cannot call cudaMalloc: a host application that embeds this
// library next to another framework whose caching allocator has already
// reserved the device memory (a new cudaMalloc there fails or fragments the
// pool), or a per-call path that cannot pay the implicit device-wide
// synchronisation of cudaMalloc/cudaFree. For them this entry point keeps
// every intermediate -- quadrature nodes, Bessel and Wigner tables, the
// per-class Q/RgQ scratch and the work descriptors -- in one file-scope
// static device array of TMX_NOALLOC_BYTES (2.25 MiB). Every GPU that loads
// the library holds that array until the process exits.
//
// Limits: nmax <= 32, ngauss <= 64. Every call shares the array and keeps the
// previous call's contents; all of it is rewritten before use, and calls
// whose work overlaps on the GPU (different streams, or different host
// threads on one device) race on it.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/tmx.h"
#include "tmx_common.cuh"
#include "tmx_kernels.h"

#define NA_MAX_NMAX 32
#define NA_MAX_NG 64
#define NA_MAX_ITEMS (4 + 2 * NA_MAX_NMAX)
#define NA_MAX_DEV 64
#define TMX_NOALLOC_BYTES (2304u * 1024u)

static constexpr size_t na_align(size_t x) { return (x + 255) & ~(size_t)255; }

// byte layout of the static array
static constexpr size_t NA_GLX = 0;
static constexpr size_t NA_GLW = na_align(NA_GLX + NA_MAX_NG * sizeof(double));
static constexpr size_t NA_GLOFF = na_align(NA_GLW + NA_MAX_NG * sizeof(double));
static constexpr size_t NA_GRAIN =
    na_align(NA_GLOFF + (NA_MAX_NG + 1) * sizeof(int64_t));
static constexpr size_t NA_SLOT = na_align(NA_GRAIN + sizeof(TmxGrain));
static constexpr size_t NA_JOB = na_align(NA_SLOT + sizeof(TmxSlot));
static constexpr size_t NA_WIGOFF = na_align(NA_JOB + sizeof(TmxWigJob));
static constexpr size_t NA_ITEMS = na_align(NA_WIGOFF + sizeof(int64_t));
static constexpr size_t NA_STATUS =
    na_align(NA_ITEMS + NA_MAX_ITEMS * sizeof(TmxItem));
static constexpr size_t NA_TAB = na_align(NA_STATUS + sizeof(int32_t));
static constexpr size_t NA_NSC =
    na_align(NA_TAB + (size_t)NA_MAX_NG * NA_MAX_NMAX * TMX_NQ * sizeof(double));
static constexpr size_t NA_WIG =
    na_align(NA_NSC + (size_t)NA_MAX_NG * TMX_NS * sizeof(double));
static constexpr size_t NA_SCR =
    na_align(NA_WIG + (size_t)(NA_MAX_NMAX + 1) * NA_MAX_NG * NA_MAX_NMAX * 2 *
                          sizeof(double));
// Q/RgQ scratch: sum over items of 2 nb^2 complex is below the complex size
// of the T-matrix itself, 4 nmax^2 + 4 sum_m (nmax + 1 - m)^2 = 49856 at 32
static constexpr size_t NA_SCR_ELEMS = 49856;
static constexpr size_t NA_END = NA_SCR + NA_SCR_ELEMS * sizeof(cplx);
static_assert(NA_END <= TMX_NOALLOC_BYTES, "static scratch layout too large");

static __device__ __align__(256) unsigned char tmx_noalloc_scratch[TMX_NOALLOC_BYTES];

struct NoallocSetup {
  TmxGrain grain;
  int32_t nmax, ngauss, nitems, pad;
  double glx[NA_MAX_NG];
  double glw[NA_MAX_NG];
  TmxItem items[NA_MAX_ITEMS];
};

// Writes the descriptors and the quadrature nodes into the static array;
// the tables and the scratch are fully rewritten by the kernels that follow.
__global__ void k_noalloc_setup(const NoallocSetup p) {
  unsigned char *base = tmx_noalloc_scratch;
  double *glx = reinterpret_cast<double *>(base + NA_GLX);
  double *glw = reinterpret_cast<double *>(base + NA_GLW);
  int64_t *gloff = reinterpret_cast<int64_t *>(base + NA_GLOFF);
  for (int i = threadIdx.x; i < NA_MAX_NG; i += blockDim.x) {
    glx[i] = (i < p.ngauss) ? p.glx[i] : 0.;
    glw[i] = (i < p.ngauss) ? p.glw[i] : 0.;
  }
  for (int i = threadIdx.x; i <= NA_MAX_NG; i += blockDim.x) {
    gloff[i] = 0;
  }
  TmxItem *items = reinterpret_cast<TmxItem *>(base + NA_ITEMS);
  for (int i = threadIdx.x; i < p.nitems; i += blockDim.x) {
    items[i] = p.items[i];
  }
  if (threadIdx.x == 0) {
    *reinterpret_cast<TmxGrain *>(base + NA_GRAIN) = p.grain;
    TmxSlot s;
    s.grain = 0;
    s.nmax = p.nmax;
    s.ngauss = p.ngauss;
    s.wig_n = 0;
    s.tab = 0;
    s.nsc = 0;
    s.tout = 0;
    s.diag = 0;
    *reinterpret_cast<TmxSlot *>(base + NA_SLOT) = s;
    TmxWigJob j;
    j.nmax = p.nmax;
    j.ngauss = p.ngauss;
    j.m_lo = 0;
    j.m_hi = p.nmax;
    j.out = 0;
    *reinterpret_cast<TmxWigJob *>(base + NA_JOB) = j;
    *reinterpret_cast<int64_t *>(base + NA_WIGOFF) = 0;
    *reinterpret_cast<int32_t *>(base + NA_STATUS) = 0;
  }
}

static std::mutex na_mutex;
static unsigned char *na_addr[NA_MAX_DEV];

// Device address of the static array on the current device, looked up once
// per device with that device current.
static int na_device_base(int dev, unsigned char **out) {
  std::lock_guard<std::mutex> lock(na_mutex);
  if (!na_addr[dev]) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, tmx_noalloc_scratch);
    if (e != cudaSuccess || ptr == nullptr) {
      fprintf(stderr, "tmx_tmatrix_fixed_noalloc: cudaGetSymbolAddress failed: %s\n",
              cudaGetErrorString(e));
      return TMX_ERR_CUDA;
    }
    na_addr[dev] = static_cast<unsigned char *>(ptr);
  }
  *out = na_addr[dev];
  return TMX_OK;
}

#define NA_CK(call)                                                            \
  do {                                                                         \
    const cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) {                                                   \
      fprintf(stderr, "tmx_tmatrix_fixed_noalloc: %s: %s\n", #call,            \
              cudaGetErrorString(e_));                                         \
      return TMX_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)

extern "C" int tmx_tmatrix_fixed_noalloc(double r_ev, double wavelength,
                                         double mr, double mi,
                                         double axis_ratio, int32_t nmax,
                                         int32_t ngauss, double *T_dev,
                                         int32_t *status_dev, void *stream) {
  if (nmax < 2 || nmax > NA_MAX_NMAX || ngauss < 1 || ngauss > NA_MAX_NG) {
    fprintf(stderr,
            "tmx_tmatrix_fixed_noalloc: nmax %d / ngauss %d outside the static "
            "scratch limits 2 <= nmax <= %d, 1 <= ngauss <= %d\n",
            nmax, ngauss, NA_MAX_NMAX, NA_MAX_NG);
    return TMX_ERR_INVALID;
  }
  if (!T_dev || !(r_ev > 0.) || !(wavelength > 0.) || !(axis_ratio > 0.) ||
      !std::isfinite(r_ev) || !std::isfinite(wavelength) ||
      !std::isfinite(axis_ratio) || !std::isfinite(mr) || !std::isfinite(mi)) {
    fprintf(stderr, "tmx_tmatrix_fixed_noalloc: invalid grain or null output\n");
    return TMX_ERR_INVALID;
  }
  int dev = 0;
  NA_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAX_DEV) {
    return TMX_ERR_NO_DEVICE;
  }
  unsigned char *base = nullptr;
  int rc = na_device_base(dev, &base);
  if (rc) {
    return rc;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  NoallocSetup p;
  memset(&p, 0, sizeof(p));
  p.grain.r_ev = r_ev;
  p.grain.k = 2. * M_PI / wavelength;
  p.grain.mr = mr;
  p.grain.mi = mi;
  p.grain.axis_ratio = axis_ratio;
  p.grain.cbrt_d = cbrt(axis_ratio);
  p.nmax = nmax;
  p.ngauss = ngauss;
  std::vector<double> x(2 * ngauss), w(2 * ngauss);
  tmx_host_gauss_legendre(2 * ngauss, x.data(), w.data());
  for (int i = 0; i < ngauss; ++i) {
    p.glx[i] = x[i];
    p.glw[i] = w[i];
  }
  int64_t scr = 0;
  int max_nb = 0;
  for (int m = 0; m <= nmax; ++m) {
    for (int c = 0; c < (m == 0 ? 4 : 2); ++c) {
      const int nb = tmx_host_class_size(nmax, m, c);
      if (nb <= 0) {
        continue;
      }
      TmxItem &it = p.items[p.nitems++];
      it.slot = 0;
      it.m = (int16_t)m;
      it.cls = (int16_t)c;
      it.scratch = scr;
      scr += 2 * (int64_t)nb * nb;
      max_nb = nb > max_nb ? nb : max_nb;
    }
  }
  if (scr > (int64_t)NA_SCR_ELEMS) {
    return TMX_ERR_INVALID;
  }

  k_noalloc_setup<<<1, 128, 0, st>>>(p);
  NA_CK(cudaGetLastError());
  tmx_launch_wigner(reinterpret_cast<const TmxWigJob *>(base + NA_JOB), 1,
                    (nmax + 1) * ngauss,
                    reinterpret_cast<const double *>(base + NA_GLX),
                    reinterpret_cast<const int64_t *>(base + NA_GLOFF),
                    reinterpret_cast<double *>(base + NA_WIG), st);
  NA_CK(cudaGetLastError());
  tmx_launch_tables(reinterpret_cast<const TmxSlot *>(base + NA_SLOT), 1,
                    reinterpret_cast<const TmxGrain *>(base + NA_GRAIN),
                    reinterpret_cast<const double *>(base + NA_GLX),
                    reinterpret_cast<const double *>(base + NA_GLW),
                    reinterpret_cast<const int64_t *>(base + NA_GLOFF),
                    reinterpret_cast<double *>(base + NA_TAB),
                    reinterpret_cast<double *>(base + NA_NSC), 800, ngauss, nmax,
                    st);
  NA_CK(cudaGetLastError());
  // structural zeros of the T blocks (entries outside each parity class)
  NA_CK(cudaMemsetAsync(T_dev, 0, tmx_tmatrix_size(nmax) * sizeof(cplx), st));
  TmxBlockArgs B;
  B.items = reinterpret_cast<const TmxItem *>(base + NA_ITEMS);
  B.nitems = p.nitems;
  B.slots = reinterpret_cast<const TmxSlot *>(base + NA_SLOT);
  B.grains = reinterpret_cast<const TmxGrain *>(base + NA_GRAIN);
  B.tab = reinterpret_cast<const double *>(base + NA_TAB);
  B.nsc = reinterpret_cast<const double *>(base + NA_NSC);
  B.wig = reinterpret_cast<const double *>(base + NA_WIG);
  B.wig_off = reinterpret_cast<const int64_t *>(base + NA_WIGOFF);
  B.scratch = reinterpret_cast<cplx *>(base + NA_SCR);
  B.tout = reinterpret_cast<cplx *>(T_dev);
  B.diag = nullptr;
  B.status = reinterpret_cast<int32_t *>(base + NA_STATUS);
  B.max_nb = max_nb;
  B.chunk_nodes = tmx_host_chunk_nodes(max_nb);
  tmx_launch_blocks(B, st);
  NA_CK(cudaGetLastError());
  // the grain's status bits (singular pivot, non-finite entries) into the
  // caller's device word: a stream-ordered copy, no allocation
  if (status_dev) {
    NA_CK(cudaMemcpyAsync(status_dev, base + NA_STATUS, sizeof(int32_t),
                          cudaMemcpyDeviceToDevice, st));
  }
  return TMX_OK;
}
