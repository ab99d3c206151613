// Device kernels of getMotion_v2's wrong-region correction
// (utils/calFlowCrossResolution.py:1190-1900, 2240-2467): the residual and
// validity of a finished pass, control-point errors, bad-region detection on
// the CP grid, and the trap mask grown in reference space.
//
// Included by wr_api.cu after wr_xres.cuh.
#pragma once

namespace wr {

// residual = 3x3 box (edge-replicated, in-plane) of It_raw, 0 where excluded;
// valid = !excluded (utils/calFlowCrossResolution.py:2101-2112)
__global__ void k_wr_residual(const float* __restrict__ it, const uint8_t* __restrict__ ex, float* __restrict__ res,
                              int nx, int ny, int nz) {
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    WR_FOR_COLS(nx, x) {
      const size_t i = (size_t)row * nx + x;
      if (ex[i]) {
        res[i] = 0.f;
        continue;
      }
      double s = 0.0;
      for (int dy = -1; dy <= 1; ++dy) {
        const float* r = it + ((size_t)z * ny + clampi(y + dy, 0, ny - 1)) * nx;
        for (int dx = -1; dx <= 1; ++dx) s += (double)r[clampi(x + dx, 0, nx - 1)];
      }
      res[i] = (float)(s * (double)(1.f / 9.f));
    }
  }
}

// err_cp = window mean of residual^2 (metric 0) or |residual| (metric 1) at
// each CP, the window edge-replicated (get_local_error_on_control_points,
// :1190-1222); one thread per CP.
__global__ void k_wr_cp_error(const float* __restrict__ res, double* __restrict__ err, int nx, int ny, int nz, int r,
                              int ncx, int ncy, int metric) {
  const long long ncp = (long long)ncx * ncy * nz;
  const int w = 2 * r + 1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ncp; i += (long long)gridDim.x * blockDim.x) {
    const int cx = (int)(i % ncx);
    const long long rest = i / ncx;
    const int cy = (int)(rest % ncy), z = (int)(rest / ncy);
    const int x0 = r + cx * w, y0 = r + cy * w;
    double s = 0.0;
    for (int dy = -r; dy <= r; ++dy) {
      const float* row = res + ((size_t)z * ny + clampi(y0 + dy, 0, ny - 1)) * nx;
      for (int dx = -r; dx <= r; ++dx) {
        const double v = row[clampi(x0 + dx, 0, nx - 1)];
        s += metric == 0 ? v * v : fabs(v);
      }
    }
    err[i] = s * (double)(1.f / (float)(w * w));
  }
}

// Median of v[0..n) (NumPy: the mean of the two middle values for even n)
// by a bitonic sort of the block's shared buffer (n <= capacity, a power of
// two); the buffer is left sorted.
__device__ double block_median(double* buf, int n, int cap) {
  for (int i = n + threadIdx.x; i < cap; i += blockDim.x) buf[i] = INFINITY;
  __syncthreads();
  for (int k = 2; k <= cap; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < cap; i += blockDim.x) {
        const int p = i ^ j;
        if (p > i) {
          const bool up = (i & k) == 0;
          const double a = buf[i], b = buf[p];
          if ((a > b) == up) { buf[i] = b; buf[p] = a; }
        }
      }
      __syncthreads();
    }
  }
  const double m = (n & 1) ? buf[n / 2] : (buf[n / 2 - 1] + buf[n / 2]) / 2.0;
  __syncthreads();
  return m;
}

// Per-slice working set of the detection: cap float64 sort keys (cap = n
// rounded up to a power of two) and 6 n ints (labels, sizes, 4 box bounds).
// Up to kWrSharedBytes it lives in shared memory, beyond in global scratch.
constexpr int kWrSharedBytes = 200 * 1024;
__host__ __device__ inline int wr_sort_cap(int n) {
  int cap = 1;
  while (cap < n) cap <<= 1;
  return cap;
}
__host__ __device__ inline size_t wr_slice_bytes(int n) {
  return ((size_t)wr_sort_cap(n) * 8 + (size_t)n * 24 + 255) & ~(size_t)255;
}

struct WrBox { int x0, x1, y0, y1, z; };

// One CTA per z slice (build_bad_region_mask_from_cp_error, :1570-1787):
// robust z-scores of the slice's CP errors (median / MAD over the inner CPs
// when the grid has more than 144), significant CPs joined 4-connected in the
// slice, components of at least min_size CPs widened by ceil(1.5 r) voxels
// to boxes (appended to boxes, count in *nbox).  gscratch null: the working
// set in dynamic shared memory; else slice z's at gscratch + z
// wr_slice_bytes(n) (grids of more control points than shared memory holds).
__global__ void k_wr_bad_regions(const double* __restrict__ err, int ncx, int ncy, int r, int nx, int ny,
                                 float mad_threshold, int min_size, WrBox* __restrict__ boxes, int* __restrict__ nbox,
                                 int max_boxes, char* __restrict__ gscratch) {
  extern __shared__ double wr_sm[];
  const int z = blockIdx.x;
  const int n = ncx * ncy;
  const int cap = wr_sort_cap(n);
  double* buf = gscratch ? reinterpret_cast<double*>(gscratch + (size_t)z * wr_slice_bytes(n)) : wr_sm;   // cap
  int* lab = reinterpret_cast<int*>(buf + cap);                     // n
  int* size = lab + n;                                              // n
  int* bb = size + n;                                               // 4 n: min x, max x, min y, max y
  __shared__ int changed;
  const double* e = err + (size_t)z * n;
  const bool inner = n > 144 && ncx > 2 && ncy > 2;
  const int sx0 = inner ? 1 : 0, sx1 = inner ? ncx - 1 : ncx, sy0 = inner ? 1 : 0, sy1 = inner ? ncy - 1 : ncy;
  const int wsub = sx1 - sx0, m = wsub * (sy1 - sy0);
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const int a = i % wsub, b = i / wsub;
    buf[i] = e[(sy0 + b) * ncx + sx0 + a];
  }
  __syncthreads();
  const double med = block_median(buf, m, cap);
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const int a = i % wsub, b = i / wsub;
    buf[i] = fabs(e[(sy0 + b) * ncx + sx0 + a] - med);
  }
  __syncthreads();
  const double mad = block_median(buf, m, cap);
  const double eps = 1e-12;
  // labels: index + 1 for significant CPs, 0 otherwise
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int a = i % ncx, b = i / ncx;
    bool sig = false;
    if (a >= sx0 && a < sx1 && b >= sy0 && b < sy1 && !(mad < eps))
      sig = fabs(e[i] - med) / (1.4826 * mad + eps) > (double)mad_threshold;
    lab[i] = sig ? i + 1 : 0;
  }
  __syncthreads();
  // 4-connected components by minimum-label propagation (at most n rounds)
  for (int round = 0; round < n; ++round) {
    if (threadIdx.x == 0) changed = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int l = lab[i];
      if (!l) continue;
      const int a = i % ncx, b = i / ncx;
      int mn = l;
      if (a > 0 && lab[i - 1]) mn = min(mn, lab[i - 1]);
      if (a + 1 < ncx && lab[i + 1]) mn = min(mn, lab[i + 1]);
      if (b > 0 && lab[i - ncx]) mn = min(mn, lab[i - ncx]);
      if (b + 1 < ncy && lab[i + ncx]) mn = min(mn, lab[i + ncx]);
      if (mn < l) {
        atomicMin(&lab[i], mn);
        changed = 1;
      }
    }
    __syncthreads();
    if (!changed) break;
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    size[i] = 0;
    bb[4 * i] = 1 << 30; bb[4 * i + 1] = -1; bb[4 * i + 2] = 1 << 30; bb[4 * i + 3] = -1;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int l = lab[i];
    if (!l) continue;
    const int root = l - 1, a = i % ncx, b = i / ncx;
    atomicAdd(&size[root], 1);
    atomicMin(&bb[4 * root], a); atomicMax(&bb[4 * root + 1], a);
    atomicMin(&bb[4 * root + 2], b); atomicMax(&bb[4 * root + 3], b);
  }
  __syncthreads();
  const int w = 2 * r + 1, dx = (int)ceil(1.5 * (double)r);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (size[i] < max(min_size, 1)) continue;
    const int k = atomicAdd(nbox, 1);
    if (k >= max_boxes) continue;
    WrBox bx;
    bx.x0 = max(0, r + bb[4 * i] * w - dx);
    bx.x1 = min(nx - 1, r + bb[4 * i + 1] * w + dx);
    bx.y0 = max(0, r + bb[4 * i + 2] * w - dx);
    bx.y1 = min(ny - 1, r + bb[4 * i + 3] * w + dx);
    bx.z = z;
    boxes[k] = bx;
  }
}

// bad = inside one of the boxes of the voxel's slice, and valid (ex null:
// the boxes alone); one CTA per box paints its rectangle into a zeroed mask.
__global__ void k_wr_paint_boxes(const WrBox* __restrict__ boxes, const uint8_t* __restrict__ ex,
                                 uint8_t* __restrict__ bad, int nx, int ny) {
  const WrBox b = boxes[blockIdx.x];
  const int w = b.x1 - b.x0 + 1, h = b.y1 - b.y0 + 1;
  for (int k = threadIdx.x; k < w * h; k += blockDim.x) {
    const int y = b.y0 + k / w, x = b.x0 + k % w;
    const size_t i = ((size_t)b.z * ny + y) * nx + x;
    bad[i] = (ex && ex[i]) ? 0 : 1;
  }
}

// "highresidual" exclusion (:2340-2355): dense = 3x3 box (edge-replicated,
// in-plane) of the error drop res0^2 - res1^2 over the pass (first iteration's
// residual minus the final one), 0 outside the bad boxes; float64.
__global__ void k_wr_error_drop(const float* __restrict__ res0, const float* __restrict__ res1,
                                const uint8_t* __restrict__ bad, double* __restrict__ dense, int nx, int ny, int nz) {
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    WR_FOR_COLS(nx, x) {
      const size_t i = (size_t)row * nx + x;
      if (!bad[i]) {
        dense[i] = 0.0;
        continue;
      }
      double s = 0.0;
      for (int dy = -1; dy <= 1; ++dy) {
        const size_t o = ((size_t)z * ny + clampi(y + dy, 0, ny - 1)) * nx;
        for (int dx = -1; dx <= 1; ++dx) {
          const size_t j = o + clampi(x + dx, 0, nx - 1);
          const double a = res0[j], b = res1[j];
          s += a * a - b * b;
        }
      }
      dense[i] = s * (double)(1.f / 9.f);
    }
  }
}

// the error drops inside the bad boxes, packed (they are sorted next)
__global__ void k_wr_gather_drop(const double* __restrict__ dense, const uint8_t* __restrict__ bad, long long n,
                                 double* __restrict__ out, int* __restrict__ count) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (bad[i]) out[atomicAdd(count, 1)] = dense[i];
}

// bad &= dense >= th, and valid
__global__ void k_wr_keep_high(uint8_t* __restrict__ bad, const double* __restrict__ dense, double th,
                               const uint8_t* __restrict__ ex, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    bad[i] = (bad[i] && dense[i] >= th && !ex[i]) ? 1 : 0;
}

// phase of a finished pass at a voxel of the iteration grid
template <int MODE>
__device__ __forceinline__ float3 wr_phase(const FieldSrc& f, const float4* phase0, int x, int y, int z, float fz0,
                                           size_t i) {
  const float3 m = eval_field<MODE>(f, x, y, z);
  if (phase0) {
    const float4 q = phase0[i];
    return make_float3(q.x + m.x, q.y + m.y, q.z + m.z);
  }
  return make_float3((float)x + m.x, (float)y + m.y, fz0 + m.z);
}

// Seeds: rint(phase) of the bad voxels inside the reference level.
// pass 0: bounding box (bbox[0..5] = min x, max x, min y, max y, min z, max z)
// pass 1: seed[(z - oz) * sy * sx + (y - oy) * sx + (x - ox)] = 1 in the ROI.
template <int MODE>
__global__ void k_wr_seeds(const FieldSrc f, const float4* __restrict__ phase0, const uint8_t* __restrict__ bad, int nx,
                           int ny, int nz, double zr, double zrh, int nxh, int nyh, int nzh, int pass,
                           int* __restrict__ bbox, uint8_t* __restrict__ seed, int ox, int oy, int oz, int sx, int sy) {
  // pass 0: each thread's box, then one set of atomics per warp (every lane
  // of a row warp reaches the end: the row loop is warp-uniform)
  int lo_x = INT_MAX, hi_x = INT_MIN, lo_y = INT_MAX, hi_y = INT_MIN, lo_z = INT_MAX, hi_z = INT_MIN;
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    const float fz0 = (float)(((double)z * zr) / zrh);
    WR_FOR_COLS(nx, x) {
      const size_t i = (size_t)row * nx + x;
      if (!bad[i]) continue;
      const float3 p = wr_phase<MODE>(f, phase0, x, y, z, fz0, i);
      const int qx = (int)rintf(p.x), qy = (int)rintf(p.y), qz = (int)rintf(p.z);
      if (qx < 0 || qx >= nxh || qy < 0 || qy >= nyh || qz < 0 || qz >= nzh) continue;
      if (pass == 0) {
        lo_x = min(lo_x, qx); hi_x = max(hi_x, qx);
        lo_y = min(lo_y, qy); hi_y = max(hi_y, qy);
        lo_z = min(lo_z, qz); hi_z = max(hi_z, qz);
      } else {
        seed[((size_t)(qz - oz) * sy + (qy - oy)) * sx + (qx - ox)] = 1;
      }
    }
  }
  if (pass != 0) return;
  lo_x = __reduce_min_sync(0xffffffffu, lo_x); hi_x = __reduce_max_sync(0xffffffffu, hi_x);
  lo_y = __reduce_min_sync(0xffffffffu, lo_y); hi_y = __reduce_max_sync(0xffffffffu, hi_y);
  lo_z = __reduce_min_sync(0xffffffffu, lo_z); hi_z = __reduce_max_sync(0xffffffffu, hi_z);
  if (threadIdx.x == 0 && hi_x >= 0) {
    atomicMin(bbox, lo_x); atomicMax(bbox + 1, hi_x);
    atomicMin(bbox + 2, lo_y); atomicMax(bbox + 3, hi_y);
    atomicMin(bbox + 4, lo_z); atomicMax(bbox + 5, hi_z);
  }
}

// Binary morphology on a (sz, sy, sx) uint8 ROI with a symmetric structuring
// element given as offsets (x, y, z); outside the ROI counts as 0 (scipy's
// border_value 0).  Rows (y, z) by blocks, x by threads: no 64-bit division.
//
// Dilation by scatter: every set voxel writes 1 at its offsets into a zeroed
// out (the work is set voxels x offsets; the sets here are sparse seeds and
// regions grown from them).
__global__ void k_wr_dilate_scatter(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int sx, int sy, int sz,
                                    const int3* __restrict__ off, int noff) {
  WR_FOR_ROWS(sz * sy, row) {
    const int z = row / sy, y = row - z * sy;
    WR_FOR_COLS(sx, x) {
      if (!in[(size_t)row * sx + x]) continue;
      for (int k = 0; k < noff; ++k) {
        const int3 o = off[k];
        const int qx = x + o.x, qy = y + o.y, qz = z + o.z;
        if (qx >= 0 && qx < sx && qy >= 0 && qy < sy && qz >= 0 && qz < sz) out[((size_t)qz * sy + qy) * sx + qx] = 1;
      }
    }
  }
}

// Erosion: a voxel stays set when every offset lands on a set voxel inside
// the ROI; the element holds (0, 0, 0), so unset voxels stay unset.
__global__ void k_wr_erode(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int sx, int sy, int sz,
                           const int3* __restrict__ off, int noff) {
  WR_FOR_ROWS(sz * sy, row) {
    const int z = row / sy, y = row - z * sy;
    WR_FOR_COLS(sx, x) {
      const size_t i = (size_t)row * sx + x;
      bool v = in[i] != 0;
      for (int k = 0; k < noff && v; ++k) {
        const int3 o = off[k];
        const int qx = x + o.x, qy = y + o.y, qz = z + o.z;
        v = qx >= 0 && qx < sx && qy >= 0 && qy < sy && qz >= 0 && qz < sz && in[((size_t)qz * sy + qy) * sx + qx];
      }
      out[i] = v ? 1 : 0;
    }
  }
}

// out &= keep; *changed set when out differs from prev (one growth step).
// 16 bytes per thread (the ROI buffers start 256-byte aligned), tail by bytes.
__global__ void k_wr_keep(uint8_t* __restrict__ out, const uint8_t* __restrict__ keep, const uint8_t* __restrict__ prev,
                          long long n, int* __restrict__ changed) {
  int c = 0;
  const long long n16 = n >> 4;
  const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, step = (long long)gridDim.x * blockDim.x;
  for (long long i = t0; i < n16; i += step) {
    uint4 o = reinterpret_cast<const uint4*>(out)[i];
    const uint4 k = reinterpret_cast<const uint4*>(keep)[i];
    const uint4 p = reinterpret_cast<const uint4*>(prev)[i];
    o.x &= k.x; o.y &= k.y; o.z &= k.z; o.w &= k.w;   // bytes are 0 / 1: AND is the logical and
    reinterpret_cast<uint4*>(out)[i] = o;
    c |= (o.x != p.x) | (o.y != p.y) | (o.z != p.z) | (o.w != p.w);
  }
  for (long long i = (n16 << 4) + t0; i < n; i += step) {
    const uint8_t v = (out[i] && keep[i]) ? 1 : 0;
    out[i] = v;
    c |= v != prev[i];
  }
  if (__any_sync(0xffffffffu, c) && (threadIdx.x & 31) == 0) atomicOr(changed, 1);
}

// scipy's "reflect" (half-sample symmetric) index of q on a line of len,
// repeating for offsets longer than the line
__device__ __forceinline__ int reflect_index(int q, int len) {
  if (q >= 0 && q < len) return q;
  const int period = 2 * len;
  q %= period;
  if (q < 0) q += period;
  return q >= len ? period - 1 - q : q;
}

// scipy.ndimage.gaussian_filter of the ROI (x0, y0, z0) + (sx, sy, sz) of a
// (., ny, nx) float32 level, evaluated only where near is set (the only
// voxels whose smoothed value is read).  It reproduces scipy's three
// correlate1d passes (x, then y, then z): mode "reflect" at the ROI's faces,
// float64 sums rounded to float32 after each pass, and correlate1d's order
// for symmetric weights: the centre term, then the tap pairs from the
// outermost inwards, (left + right) w, with no fused multiply-add.
// w points at the centre weight, w[j] = the weight at offsets -j and +j;
// rad < 0: no smoothing (sigma 0), the crop itself.
struct GaussRoi {
  const float* lev;
  int nx, ny, x0, y0, z0, sx, sy, sz, rad;
  const double* w;
};

__device__ __forceinline__ float gauss_x(const GaussRoi& g, int x, int y, int z) {
  const float* line = g.lev + ((size_t)(z + g.z0) * g.ny + (y + g.y0)) * g.nx + g.x0;
  double s = __dmul_rn((double)line[x], g.w[0]);
  for (int j = g.rad; j >= 1; --j)
    s = __dadd_rn(s, __dmul_rn(__dadd_rn((double)line[reflect_index(x - j, g.sx)],
                                         (double)line[reflect_index(x + j, g.sx)]), g.w[j]));
  return (float)s;
}

__device__ __forceinline__ float gauss_xy(const GaussRoi& g, int x, int y, int z) {
  double s = __dmul_rn((double)gauss_x(g, x, y, z), g.w[0]);
  for (int j = g.rad; j >= 1; --j)
    s = __dadd_rn(s, __dmul_rn(__dadd_rn((double)gauss_x(g, x, reflect_index(y - j, g.sy), z),
                                         (double)gauss_x(g, x, reflect_index(y + j, g.sy), z)), g.w[j]));
  return (float)s;
}

// One full correlate1d pass of the same filter along AXIS (0 x, 1 y, 2 z)
// over a contiguous (sz, sy, sx) float32 ROI (src_nx / src_ny / offsets:
// where the input lives; the first pass reads the level, later ones the
// previous pass), in the order and rounding of gauss_x.
template <int AXIS>
__global__ void k_wr_gauss_pass(const float* __restrict__ src, int src_nx, int src_ny, int x0, int y0, int z0,
                                float* __restrict__ out, int sx, int sy, int sz, const double* __restrict__ w, int rad) {
  WR_FOR_ROWS(sz * sy, row) {
    const int z = row / sy, y = row - z * sy;
    const float* base = src + ((size_t)(z + z0) * src_ny + (y + y0)) * src_nx + x0;
    const size_t stride = AXIS == 0 ? 1 : AXIS == 1 ? (size_t)src_nx : (size_t)src_nx * src_ny;
    const int c = AXIS == 1 ? y : z;
    const int len = AXIS == 0 ? sx : AXIS == 1 ? sy : sz;
    WR_FOR_COLS(sx, x) {
      const float* p = base + x;
      const int cc = AXIS == 0 ? x : c;
      const float* line = p - (size_t)cc * stride;
      double s = __dmul_rn((double)*p, w[0]);
      for (int j = rad; j >= 1; --j)
        s = __dadd_rn(s, __dmul_rn(__dadd_rn((double)line[(size_t)reflect_index(cc - j, len) * stride],
                                             (double)line[(size_t)reflect_index(cc + j, len) * stride]), w[j]));
      out[(size_t)row * sx + x] = (float)s;
    }
  }
}

__global__ void k_wr_gauss_near(const GaussRoi g, const uint8_t* __restrict__ near, float* __restrict__ out) {
  WR_FOR_ROWS(g.sz * g.sy, row) {
    const int z = row / g.sy, y = row - z * g.sy;
    WR_FOR_COLS(g.sx, x) {
      const size_t i = (size_t)row * g.sx + x;
      if (!near[i]) continue;
      if (g.rad < 0) {
        out[i] = g.lev[((size_t)(z + g.z0) * g.ny + (y + g.y0)) * g.nx + g.x0 + x];
        continue;
      }
      double s = __dmul_rn((double)gauss_xy(g, x, y, z), g.w[0]);
      for (int j = g.rad; j >= 1; --j)
        s = __dadd_rn(s, __dmul_rn(__dadd_rn((double)gauss_xy(g, x, y, reflect_index(z - j, g.sz)),
                                             (double)gauss_xy(g, x, y, reflect_index(z + j, g.sz))), g.w[j]));
      out[i] = (float)s;
    }
  }
}

// the ROI's values under the seed mask, packed (order irrelevant: they are sorted)
__global__ void k_wr_gather(const float* __restrict__ v, const uint8_t* __restrict__ m, long long n,
                            float* __restrict__ out, int* __restrict__ count) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (m[i]) out[atomicAdd(count, 1)] = v[i];
}

// |v - med| in float32 (a float32 array minus a Python float)
__global__ void k_wr_absdev(const float* __restrict__ v, int n, float med, float* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = fabsf(v[i] - med);
}

// allowed = (near & |sm - med| <= tol) | seed, all float32 comparisons
__global__ void k_wr_allowed(const float* __restrict__ sm, const uint8_t* __restrict__ near,
                             const uint8_t* __restrict__ seed, long long n, float med, float tol,
                             uint8_t* __restrict__ allowed) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    allowed[i] = ((near[i] && fabsf(sm[i] - med) <= tol) || seed[i]) ? 1 : 0;
}

// corrected = level mask | region pasted at the ROI origin
__global__ void k_wr_paste(const uint8_t* __restrict__ region, uint8_t* __restrict__ mask, int nxh, int nyh,
                           int ox, int oy, int oz, int sx, int sy, int sz) {
  const long long n = (long long)sx * sy * sz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (!region[i]) continue;
    const int x = (int)(i % sx);
    const long long rest = i / sx;
    const int y = (int)(rest % sy), z = (int)(rest / sy);
    mask[((size_t)(z + oz) * nyh + (y + oy)) * nxh + (x + ox)] = 1;
  }
}

// valid voxels under a reference mask spline: !moving-excluded and
// H_mask(phase) <= 0.5 (compute_valid_mask_on_moving_grid, :2006-2028)
template <int MODE>
__global__ void k_wr_count_valid(const FieldSrc f, const float4* __restrict__ phase0, const uint8_t* __restrict__ mbits,
                                 const double* __restrict__ cmask, const float2* __restrict__ cbounds, int pxh,
                                 int pyh, int pzh, int nx, int ny, int nz,
                                 double zr, double zrh, unsigned long long* __restrict__ count) {
  unsigned long long c = 0;
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    const float fz0 = (float)(((double)z * zr) / zrh);
    WR_FOR_COLS(nx, x) {
      const size_t i = (size_t)row * nx + x;
      if (mbits && (mbits[i] & 1)) continue;
      const float3 p = wr_phase<MODE>(f, phase0, x, y, z, fz0, i);
      if (!mask_above_half(cmask, cbounds, pxh, pyh, pzh, p.x, p.y, p.z)) ++c;
    }
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

__global__ void k_wr_count_u8(const uint8_t* __restrict__ v, long long n, int want, unsigned long long* __restrict__ count) {
  unsigned long long c = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    c += ((v[i] != 0) == (want != 0)) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// Error of a finished pass (the final recompute, :2211-2216): mean of the
// residual squared (errpart: per-tile sums of the eval launch) plus the
// smoothness penalty of the CP neighbour differences without z scaling.
__global__ void k_wr_pass_error(const double* __restrict__ errpart, long long nblk, const float4* __restrict__ cp,
                                int ncx, int ncy, int nz, double sps, double n_vox, double* __restrict__ out) {
  __shared__ double red[2][256];
  double e = 0.0, pen = 0.0;
  for (long long i = threadIdx.x; i < nblk; i += blockDim.x) e += errpart[i];
  const long long ncp = (long long)ncx * ncy * nz;
  for (long long i = threadIdx.x; i < ncp; i += blockDim.x) {
    const int cx = (int)(i % ncx);
    const long long rest = i / ncx;
    const int cy = (int)(rest % ncy), z = (int)(rest / ncy);
    const float4* b = cp + (size_t)z * ncy * ncx;
    double sx = 0.0, sy = 0.0, szz = 0.0;
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        if (dx == 0 && dy == 0) continue;
        const float4 v = b[clampi(cy + dy, 0, ncy - 1) * ncx + clampi(cx + dx, 0, ncx - 1)];
        sx += 0.125 * (double)v.x;
        sy += 0.125 * (double)v.y;
        szz += 0.125 * (double)v.z;
      }
    const float4 c = b[cy * ncx + cx];
    const float ndx = (float)(sx - (double)c.x), ndy = (float)(sy - (double)c.y), ndz = (float)(szz - (double)c.z);
    pen += (double)(ndx * ndx + ndy * ndy + ndz * ndz);
  }
  red[0][threadIdx.x] = e;
  red[1][threadIdx.x] = pen;
  __syncthreads();
  for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
    if (threadIdx.x < s2) {
      red[0][threadIdx.x] += red[0][threadIdx.x + s2];
      red[1][threadIdx.x] += red[1][threadIdx.x + s2];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0][0] / n_vox + red[1][0] * sps / n_vox;
}

__global__ void k_wr_set_active(LKState* st) { st->active = 1; }

// a re-run of a level: fresh stopping state, the level's log kept
__global__ void k_wr_pass_begin(LKState* st, int level) {
  st->active = 1;
  st->do_update = 0;
  st->level = level;
  st->n_updates = 0;
  st->maxdiff_bits = 0u;
  st->old_err[0] = st->old_err[1] = st->old_err[2] = INFINITY;
}

}  // namespace wr
