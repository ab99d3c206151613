// Outlier masks of the per-batch registration wrapper (utils/mask.py):
// getMask (robust z-score threshold, (3,3,1) opening, (3,3,1) dilation) and
// bwareafilt3_wei (26-connected components kept by size), on the device.
//
// Layout: volumes are (z, y, x) with x fastest; the reference's (x, y, z)
// arrays are the same memory, so its (3,3,1) footprint is a 3x3 square in
// each z slice here, and 26-connectivity is symmetric in the axes.

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <string>

#include "wr_b200.h"
#include "wr_mask.h"

namespace wrmask {

static thread_local std::string g_err;
static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

constexpr int kThreads = 256;
constexpr int kRadixBits = 11;
constexpr int kRadixBins = 1 << kRadixBits;   // 2048
constexpr int kUnionIterLimit = 1 << 22;       // bound of one union's retry loop

static int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  const long long cap = 148LL * 16;
  if (b < 1) b = 1;
  return (int)(b < cap ? b : cap);
}

static size_t align_up(size_t v, size_t a = 256) { return (v + a - 1) / a * a; }

template <typename T> __device__ __forceinline__ float as_f32(const T* p, long long i) { return (float)__ldg(p + i); }

// float32 -> uint32 with the same order (radix-select keys), and back
__device__ __forceinline__ uint32_t f32_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_f32(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// ---------------------------------------------------------------------------
// exact order statistic: three radix passes (bits 21..31, 10..20, 0..9) over
// the keys that share the prefix found so far
// ---------------------------------------------------------------------------

struct SelectState {
  uint32_t prefix;       // key bits found so far
  uint32_t prefix_mask;
  long long rank;        // rank still to find among the keys matching prefix
  int shift;             // lowest bit of the current digit
  int bits;              // width of the current digit
};

template <typename T>
__global__ void k_radix_hist(const T* __restrict__ v, long long n, const SelectState* __restrict__ ss,
                             unsigned long long* __restrict__ hist) {
  __shared__ unsigned int h[kRadixBins];
  for (int i = threadIdx.x; i < kRadixBins; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const SelectState s = *ss;
  const uint32_t dmask = (1u << s.bits) - 1u;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const uint32_t k = f32_key(as_f32<T>(v, i));
    if ((k & s.prefix_mask) == s.prefix) atomicAdd(&h[(k >> s.shift) & dmask], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kRadixBins; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
}

// one block: pick the digit holding the rank, narrow the prefix, clear the
// histogram for the next pass; after the last pass write the value
__global__ void k_radix_pick(SelectState* ss, unsigned long long* hist, float* out_value) {
  if (threadIdx.x == 0) {
    SelectState s = *ss;
    const int nb = 1 << s.bits;
    long long r = s.rank;
    int d = 0;
    for (; d < nb - 1; ++d) {
      const long long c = (long long)hist[d];
      if (r < c) break;
      r -= c;
    }
    s.prefix |= (uint32_t)d << s.shift;
    s.prefix_mask |= (uint32_t)(nb - 1) << s.shift;
    s.rank = r;
    if (s.shift == 32 - kRadixBits) {
      s.shift = 32 - 2 * kRadixBits;
      s.bits = kRadixBits;
    } else if (s.shift > 0) {
      s.bits = s.shift;
      s.shift = 0;
    } else {
      s.bits = 0;
    }
    *ss = s;
    if (s.prefix_mask == 0xffffffffu && out_value) *out_value = key_f32(s.prefix);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kRadixBins; i += blockDim.x) hist[i] = 0ull;
}

__global__ void k_select_init(SelectState* ss, long long rank) {
  SelectState s;
  s.prefix = 0;
  s.prefix_mask = 0;
  s.rank = rank;
  s.bits = kRadixBits;
  s.shift = 32 - kRadixBits;
  *ss = s;
}

// ---------------------------------------------------------------------------
// robust statistics and the thresholded z-score mask
// ---------------------------------------------------------------------------

// numpy's percentile ("linear" method) of float32 data from its two order
// statistics: q = pct / 100 in float32, virtual index (n - 1) * q in float32,
// gamma = its fractional part, then numpy's two-sided lerp in float32.
__global__ void k_percentile_value(const float* __restrict__ ord, float q_pct, long long n, float* thr) {
  const float q = __fdiv_rn(q_pct, 100.f);
  const float vi = __fmul_rn((float)(n - 1), q);
  const float prev = floorf(vi);
  const float gamma = __fsub_rn(vi, prev);
  const float a = ord[0], b = ord[1];
  if (vi >= (float)(n - 1)) {
    *thr = ord[1];
    return;
  }
  const float d = __fsub_rn(b, a);
  *thr = gamma >= 0.5f ? __fsub_rn(b, __fmul_rn(d, __fsub_rn(1.f, gamma))) : __fadd_rn(a, __fmul_rn(d, gamma));
}

// Sums over the selected values (<= threshold) go to per-block partials,
// reduced in a fixed order by one block, so the statistics (and the mask)
// are the same on every run.
template <typename T>
__global__ void k_sel_sum(const T* __restrict__ v, long long n, const float* __restrict__ thr,
                          double* __restrict__ part) {
  __shared__ double red[2][kThreads];
  const float t = *thr;
  double s = 0.0, c = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float x = as_f32<T>(v, i);
    if (x <= t) { s += (double)x; c += 1.0; }
  }
  red[0][threadIdx.x] = s;
  red[1][threadIdx.x] = c;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[0][threadIdx.x] += red[0][threadIdx.x + o];
      red[1][threadIdx.x] += red[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = red[0][0];
    part[3 * blockIdx.x + 1] = red[1][0];
  }
}

// one block: total of partial column `col`, blocks in order
__device__ double sum_partials(const double* part, int nblk, int col) {
  __shared__ double red[kThreads];
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += part[3 * b + col];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

__global__ void k_sel_mean(const double* part, int nblk, double* acc) {
  const double s = sum_partials(part, nblk, 0);
  const double c = sum_partials(part, nblk, 1);
  if (threadIdx.x == 0) {
    acc[0] = s;
    acc[1] = c;
  }
}

template <typename T>
__global__ void k_sel_var(const T* __restrict__ v, long long n, const float* __restrict__ thr,
                          const double* __restrict__ acc, double* __restrict__ part) {
  __shared__ double red[kThreads];
  const float t = *thr;
  const double mean = acc[0] / acc[1];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float x = as_f32<T>(v, i);
    if (x <= t) {
      const double d = (double)x - mean;
      s += d * d;
    }
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[3 * blockIdx.x + 2] = red[0];
}

// mu, sigma as float32 (numpy's float32 mean / std of the selected values);
// stats_out: mu, sigma, percentile value as doubles
__global__ void k_stats_final(const double* part, int nblk, const double* acc, const float* thr, float* musig,
                              double* stats_out) {
  const double ss = sum_partials(part, nblk, 2);
  if (threadIdx.x == 0) {
    musig[0] = (float)(acc[0] / acc[1]);
    musig[1] = (float)sqrt(ss / acc[1]);
    if (stats_out) {
      stats_out[0] = (double)musig[0];
      stats_out[1] = (double)musig[1];
      stats_out[2] = (double)*thr;
    }
  }
}

// |(x - mu) / sigma| > thres in float32
template <typename T>
__global__ void k_zmask(const T* __restrict__ v, long long n, const float* __restrict__ musig, float thres,
                        uint8_t* __restrict__ m) {
  const float mu = musig[0], sg = musig[1];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m[i] = fabsf(__fdiv_rn(__fsub_rn(as_f32<T>(v, i), mu), sg)) > thres ? 1 : 0;
}

// 3x3 erosion in each z slice, the outside of the slice counting as set
// (binary_erosion with border_value True)
__global__ void k_erode3(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int nz, int ny, int nx) {
  const long long n = (long long)nz * ny * nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const int y = (int)((i / nx) % ny);
    uint8_t v = 1;
    for (int dy = -1; dy <= 1 && v; ++dy) {
      if (y + dy < 0 || y + dy >= ny) continue;
      for (int dx = -1; dx <= 1; ++dx) {
        if (x + dx < 0 || x + dx >= nx) continue;
        if (!in[i + (long long)dy * nx + dx]) { v = 0; break; }
      }
    }
    out[i] = v;
  }
}

// (2h+1) x (2h+1) dilation in each z slice, the outside counting as clear
// (binary_dilation with border_value False; two 3x3 dilations are one 5x5
// inside the slice)
__global__ void k_dilate(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int nz, int ny, int nx, int h) {
  const long long n = (long long)nz * ny * nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const int y = (int)((i / nx) % ny);
    uint8_t v = 0;
    for (int dy = -h; dy <= h && !v; ++dy) {
      if (y + dy < 0 || y + dy >= ny) continue;
      for (int dx = -h; dx <= h; ++dx) {
        if (x + dx < 0 || x + dx >= nx) continue;
        if (in[i + (long long)dy * nx + dx]) { v = 1; break; }
      }
    }
    out[i] = v;
  }
}

// ---------------------------------------------------------------------------
// 26-connected components: lock-free union-find on voxel indexes (each
// component's root is its smallest voxel index), then sizes and the filter
// ---------------------------------------------------------------------------

__device__ __forceinline__ int uf_find(int* L, int x) {
  int p = L[x];
  while (p != x) {
    const int g = L[p];
    if (g != p) L[x] = g;   // path halving; labels only decrease towards the root
    x = p;
    p = L[x];
  }
  return x;
}

__device__ __forceinline__ void uf_union(int* L, int a, int b, int* err) {
  for (int it = 0; it < kUnionIterLimit; ++it) {
    a = uf_find(L, a);
    b = uf_find(L, b);
    if (a == b) return;
    if (a < b) { const int t = a; a = b; b = t; }
    const int old = atomicMin(&L[a], b);
    if (old == a) return;   // a was a root and now points to b
    a = old;                // a was relinked meanwhile: retry from its new parent
  }
  atomicOr(err, 1);
}

__global__ void k_cc_init(const uint8_t* __restrict__ m, int* __restrict__ L, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    L[i] = m[i] ? (int)i : -1;
}

// union with the 13 neighbours that precede the voxel in (z, y, x) order
__global__ void k_cc_union(const uint8_t* __restrict__ m, int* L, int nz, int ny, int nx, int* err) {
  const long long n = (long long)nz * ny * nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (!m[i]) continue;
    const int x = (int)(i % nx);
    const long long r = i / nx;
    const int y = (int)(r % ny), z = (int)(r / ny);
    for (int dz = -1; dz <= 0; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          if (dz == 0 && (dy > 0 || (dy == 0 && dx >= 0))) continue;
          const int zz = z + dz, yy = y + dy, xx = x + dx;
          if (zz < 0 || yy < 0 || yy >= ny || xx < 0 || xx >= nx) continue;
          const long long j = ((long long)zz * ny + yy) * nx + xx;
          if (m[j]) uf_union(L, (int)i, (int)j, err);
        }
  }
}

// Each voxel's label becomes its root.  The walk to the root writes nothing:
// a path-halving store racing with another thread's root store could put a
// non-root ancestor back into that thread's label after the root went in,
// and the filter reads the label as the root.  Root stores alone keep every
// chain an ancestor chain.
__global__ void k_cc_flatten_count(int* L, int* __restrict__ count, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (L[i] < 0) continue;
    int root = (int)i;
    for (int q = L[root]; q != root; q = L[root]) root = q;
    L[i] = root;
    atomicAdd(&count[root], 1);
  }
}

__global__ void k_cc_filter(const int* __restrict__ L, const int* __restrict__ count, long long n, long long lo,
                            long long hi, uint8_t* __restrict__ out, int* kept) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int root = L[i];
    uint8_t keep = 0;
    if (root >= 0) {
      const long long c = count[root];
      keep = (c >= lo && c <= hi) ? 1 : 0;
      if (keep && root == (int)i) atomicAdd(kept, 1);
    }
    out[i] = keep;
  }
}

// ---------------------------------------------------------------------------
// workspace layout
// ---------------------------------------------------------------------------

struct MaskWs {
  size_t sel, hist, ord, thr, acc, part, musig, tmp, total;
};
static MaskWs mask_ws(long long n) {
  MaskWs w;
  size_t c = 0;
  w.sel = c; c = align_up(c + sizeof(SelectState));
  w.hist = c; c = align_up(c + sizeof(unsigned long long) * kRadixBins);
  w.ord = c; c = align_up(c + 2 * sizeof(float));
  w.thr = c; c = align_up(c + sizeof(float));
  w.acc = c; c = align_up(c + 2 * sizeof(double));
  w.part = c; c = align_up(c + 3 * sizeof(double) * (size_t)grid_for(n));
  w.musig = c; c = align_up(c + 2 * sizeof(float));
  w.tmp = c; c = align_up(c + (size_t)n);
  w.total = c;
  return w;
}
struct CcWs {
  size_t labels, count, kept, err, total;
};
static CcWs cc_ws(long long n) {
  CcWs w;
  size_t c = 0;
  w.labels = c; c = align_up(c + 4 * (size_t)n);
  w.count = c; c = align_up(c + 4 * (size_t)n);
  w.kept = c; c = align_up(c + sizeof(int));
  w.err = c; c = align_up(c + sizeof(int));
  w.total = c;
  return w;
}

template <typename T> static T* at(void* base, size_t off) {
  return reinterpret_cast<T*>(static_cast<char*>(base) + off);
}

template <typename T>
static void order_stat(const T* v, long long n, long long rank, void* ws, const MaskWs& W, float* out,
                       cudaStream_t s) {
  SelectState* ss = at<SelectState>(ws, W.sel);
  unsigned long long* hist = at<unsigned long long>(ws, W.hist);
  k_select_init<<<1, 1, 0, s>>>(ss, rank);
  for (int pass = 0; pass < 3; ++pass) {
    k_radix_hist<T><<<grid_for(n), kThreads, 0, s>>>(v, n, ss, hist);
    k_radix_pick<<<1, kThreads, 0, s>>>(ss, hist, pass == 2 ? out : nullptr);
  }
}

template <typename T>
static void get_mask(const T* v, int nz, int ny, int nx, double thres, double pct, uint8_t* out, double* stats_out,
                     void* ws, cudaStream_t s) {
  const long long n = (long long)nz * ny * nx;
  const MaskWs W = mask_ws(n);
  cudaMemsetAsync(at<unsigned long long>(ws, W.hist), 0, sizeof(unsigned long long) * kRadixBins, s);
  // the two order statistics around numpy's float32 virtual index (host
  // float32 arithmetic, the same operations as k_percentile_value)
  const float q = (float)pct / 100.f;
  const float vi = (float)(n - 1) * q;
  long long prev = (long long)floorf(vi);
  if (prev > n - 1) prev = n - 1;
  if (prev < 0) prev = 0;
  const long long next = prev + 1 < n ? prev + 1 : n - 1;
  float* ord = at<float>(ws, W.ord);
  order_stat<T>(v, n, prev, ws, W, ord, s);
  order_stat<T>(v, n, next, ws, W, ord + 1, s);
  float* thr = at<float>(ws, W.thr);
  k_percentile_value<<<1, 1, 0, s>>>(ord, (float)pct, n, thr);
  double* acc = at<double>(ws, W.acc);
  double* part = at<double>(ws, W.part);
  const int g = grid_for(n);
  k_sel_sum<T><<<g, kThreads, 0, s>>>(v, n, thr, part);
  k_sel_mean<<<1, kThreads, 0, s>>>(part, g, acc);
  k_sel_var<T><<<g, kThreads, 0, s>>>(v, n, thr, acc, part);
  float* musig = at<float>(ws, W.musig);
  k_stats_final<<<1, kThreads, 0, s>>>(part, g, acc, thr, musig, stats_out);
  uint8_t* tmp = at<uint8_t>(ws, W.tmp);
  k_zmask<T><<<g, kThreads, 0, s>>>(v, n, musig, (float)thres, out);
  k_erode3<<<g, kThreads, 0, s>>>(out, tmp, nz, ny, nx);
  k_dilate<<<g, kThreads, 0, s>>>(tmp, out, nz, ny, nx, 2);
}

// ---------------------------------------------------------------------------
// frame correlation of pick_initial_reference (utils/reference.py:60-78):
// per-frame means, then the demeaned Gram matrix, both accumulated in float64
// in a fixed order (deterministic).  One block per frame / per frame pair.
// ---------------------------------------------------------------------------

constexpr int kGramThreads = 256;

__device__ __forceinline__ double block_sum_d(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  return t;   // valid in thread 0
}

__global__ void __launch_bounds__(kGramThreads) k_frame_means(const float* __restrict__ x, long long d,
                                                             double* __restrict__ means) {
  __shared__ double red[kGramThreads / 32];
  const float* row = x + (long long)blockIdx.x * d;
  double s = 0.0;
  for (long long k = threadIdx.x; k < d; k += blockDim.x) s += (double)row[k];
  const double t = block_sum_d(s, red);
  if (threadIdx.x == 0) means[blockIdx.x] = t / (double)d;
}

// pair p = (i, j), j >= i, enumerated row by row
__global__ void __launch_bounds__(kGramThreads) k_frame_gram(const float* __restrict__ x, int t, long long d,
                                                            const double* __restrict__ means,
                                                            double* __restrict__ gram) {
  __shared__ double red[kGramThreads / 32];
  int i = 0, p = blockIdx.x;
  while (p >= t - i) {
    p -= t - i;
    ++i;
  }
  const int j = i + p;
  const float* a = x + (long long)i * d;
  const float* b = x + (long long)j * d;
  const double ma = means[i], mb = means[j];
  double s = 0.0;
  for (long long k = threadIdx.x; k < d; k += blockDim.x) s += ((double)a[k] - ma) * ((double)b[k] - mb);
  const double v = block_sum_d(s, red);
  if (threadIdx.x == 0) {
    gram[(long long)i * t + j] = v;
    gram[(long long)j * t + i] = v;
  }
}

}  // namespace wrmask

using namespace wrmask;

extern "C" {

const char* wr_mask_last_error(void) { return g_err.c_str(); }

int wr_mask_workspace_size(int32_t nz, int32_t ny, int32_t nx, size_t* bytes) {
  if (!bytes) return fail(WR_E_NULL, "bytes is NULL");
  if (nz < 1 || ny < 1 || nx < 1) return fail(WR_E_SHAPE, "empty volume");
  const long long n = (long long)nz * ny * nx;
  if (n >= (1LL << 31)) return fail(WR_E_SHAPE, "volume holds 2^31 voxels or more");
  const MaskWs a = mask_ws(n);
  const CcWs b = cc_ws(n);
  *bytes = a.total > b.total ? a.total : b.total;
  return 0;
}

int wr_get_mask(const WrVolume* vol, double thres_factor, double percentile, uint8_t* mask_out, double* stats_out,
                void* workspace, size_t workspace_bytes, void* stream) {
  if (!vol || !vol->data || !mask_out || !workspace) return fail(WR_E_NULL, "vol, mask_out or workspace is NULL");
  size_t need = 0;
  int rc = wr_mask_workspace_size(vol->nz, vol->ny, vol->nx, &need);
  if (rc) return rc;
  if (workspace_bytes < need) return fail(WR_E_WORKSPACE, "workspace smaller than wr_mask_workspace_size");
  if (reinterpret_cast<uintptr_t>(workspace) % 256) return fail(WR_E_WORKSPACE, "workspace must be 256-byte aligned");
  if (!(percentile >= 0.0 && percentile <= 100.0)) return fail(WR_E_PARAM, "percentile must be in [0, 100]");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (vol->dtype) {
    case WR_U16:
      get_mask<uint16_t>((const uint16_t*)vol->data, vol->nz, vol->ny, vol->nx, thres_factor, percentile, mask_out,
                         stats_out, workspace, s);
      break;
    case WR_U8:
      get_mask<uint8_t>((const uint8_t*)vol->data, vol->nz, vol->ny, vol->nx, thres_factor, percentile, mask_out,
                        stats_out, workspace, s);
      break;
    case WR_F32:
      get_mask<float>((const float*)vol->data, vol->nz, vol->ny, vol->nx, thres_factor, percentile, mask_out,
                      stats_out, workspace, s);
      break;
    default:
      return fail(WR_E_DTYPE, "dtype must be WR_U8, WR_U16 or WR_F32");
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(-(int)e, cudaGetErrorString(e));
  return 0;
}

int wr_bwareafilt3(const uint8_t* mask_in, int32_t nz, int32_t ny, int32_t nx, int64_t min_size, int64_t max_size,
                   uint8_t* mask_out, int32_t* n_components, int32_t* error_flag, void* workspace,
                   size_t workspace_bytes, void* stream) {
  if (!mask_in || !mask_out || !workspace) return fail(WR_E_NULL, "mask_in, mask_out or workspace is NULL");
  size_t need = 0;
  int rc = wr_mask_workspace_size(nz, ny, nx, &need);
  if (rc) return rc;
  if (workspace_bytes < need) return fail(WR_E_WORKSPACE, "workspace smaller than wr_mask_workspace_size");
  if (reinterpret_cast<uintptr_t>(workspace) % 256) return fail(WR_E_WORKSPACE, "workspace must be 256-byte aligned");
  if (mask_in == mask_out) return fail(WR_E_PARAM, "mask_in and mask_out must differ");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long n = (long long)nz * ny * nx;
  const CcWs W = cc_ws(n);
  int* L = at<int>(workspace, W.labels);
  int* count = at<int>(workspace, W.count);
  int* kept = at<int>(workspace, W.kept);
  int* err = at<int>(workspace, W.err);
  cudaMemsetAsync(count, 0, 4 * (size_t)n, s);
  cudaMemsetAsync(kept, 0, sizeof(int), s);
  cudaMemsetAsync(err, 0, sizeof(int), s);
  const int g = grid_for(n);
  k_cc_init<<<g, kThreads, 0, s>>>(mask_in, L, n);
  k_cc_union<<<g, kThreads, 0, s>>>(mask_in, L, nz, ny, nx, err);
  k_cc_flatten_count<<<g, kThreads, 0, s>>>(L, count, n);
  k_cc_filter<<<g, kThreads, 0, s>>>(L, count, n, (long long)min_size, (long long)max_size, mask_out, kept);
  if (n_components) cudaMemcpyAsync(n_components, kept, sizeof(int), cudaMemcpyDeviceToDevice, s);
  if (error_flag) cudaMemcpyAsync(error_flag, err, sizeof(int), cudaMemcpyDeviceToDevice, s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(-(int)e, cudaGetErrorString(e));
  return 0;
}

int wr_frame_gram(const float* frames, int32_t t, int64_t d, double* means, double* gram, void* stream) {
  if (!frames || !means || !gram) return fail(WR_E_NULL, "a required pointer is NULL");
  if (t < 1 || t > 4096 || d < 1) return fail(WR_E_SHAPE, "need 1 <= t <= 4096 frames of d >= 1 values");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_frame_means<<<t, kGramThreads, 0, s>>>(frames, d, means);
  const long long pairs = (long long)t * (t + 1) / 2;
  k_frame_gram<<<(unsigned)pairs, kGramThreads, 0, s>>>(frames, t, d, means, gram);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(-(int)e, cudaGetErrorString(e));
  return 0;
}

}  // extern "C"
