// Device code of the cross-resolution registration (getMotion_v2 of
// utils/calFlowCrossResolution.py:2470-2663 with the wrong-region correction
// off): the reference stack lives on its own grid and is read through a cubic
// B-spline ("H", :463-478), the moving stack on the iteration grid.
//
// Included by wr_api.cu after wr_kernels.cuh.
#pragma once

namespace wr {

// ---------------------------------------------------------------------------
// cubic B-spline coefficients (map_coordinates(order=3, mode="nearest"))
// ---------------------------------------------------------------------------

// SciPy and CuPy pad the input by 12 edge copies on every side before the
// prefilter when mode is "nearest"; samples address the padded coefficients.
constexpr int kSplinePad = 12;

// Edge-padded copy in float64; thresh >= 0 stores (value > thresh) as 0 / 1.
template <typename T>
__global__ void k_spline_pad(const T* __restrict__ in, double* __restrict__ out, int nx, int ny, int nz, double thresh) {
  const int px = nx + 2 * kSplinePad, py = ny + 2 * kSplinePad, pz = nz + 2 * kSplinePad;
  const long long n = (long long)px * py * pz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % px);
    const long long rest = i / px;
    const int y = (int)(rest % py), z = (int)(rest / py);
    const int sx = clampi(x - kSplinePad, 0, nx - 1), sy = clampi(y - kSplinePad, 0, ny - 1);
    const int sz = clampi(z - kSplinePad, 0, nz - 1);
    double v = (double)in[((size_t)sz * ny + sy) * nx + sx];
    if (thresh >= 0.0) v = v > thresh ? 1.0 : 0.0;
    out[i] = v;
  }
}

// Cubic B-spline prefilter (Unser's recursive filter): gain 6, a causal
// recursion c+[k] = 6 s[k] + z c+[k-1] and an anti-causal one
// c-[k] = z (c-[k+1] - c+[k]) with the pole z = sqrt(3) - 2, both started as
// if the line continued with its end values:
//   c+[0] = 6 s[0] / (1 - z),
//   c-[n-1] = -z (6 s[n-1] / (1 - z)^2 + (c+[n-1] - 6 s[n-1] / (1 - z)) / (1 - z^2)).
constexpr double kSplineZ = -0.26794919243112270;   // sqrt(3) - 2

__device__ __forceinline__ double spline_tail(double c_last, double s_end6) {
  const double z = kSplineZ;
  return -z * (s_end6 / ((1.0 - z) * (1.0 - z)) + (c_last - s_end6 / (1.0 - z)) / (1.0 - z * z));
}

// x lines (contiguous rows of n), one warp per row, in place: both
// recursions as warp scans of 32-element chunks (c_l = u_l + z c_{l-1} by
// five shuffle steps, then the carry of the previous chunk times z^(l+1)).
__global__ void k_spline_rows(double* __restrict__ c, long long nrows, int n) {
  const double z = kSplineZ;
  const long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= nrows) return;   // whole warps leave together
  double* p = c + row * (long long)n;
  double zl = z;              // z^(lane + 1)
  for (int i = 0; i < lane; ++i) zl *= z;
  const double z2 = z * z, z4 = z2 * z2, z8 = z4 * z4, z16 = z8 * z8;
  const double s_end6 = 6.0 * p[n - 1];
  double carry = 0.0;
  for (int b = 0; b < n; b += 32) {
    const int k = b + lane;
    double v = k < n ? 6.0 * p[k] : 0.0;
    if (k == 0) v = v / (1.0 - z);
    double t = __shfl_up_sync(0xffffffffu, v, 1);
    if (lane >= 1) v = fma(z, t, v);
    t = __shfl_up_sync(0xffffffffu, v, 2);
    if (lane >= 2) v = fma(z2, t, v);
    t = __shfl_up_sync(0xffffffffu, v, 4);
    if (lane >= 4) v = fma(z4, t, v);
    t = __shfl_up_sync(0xffffffffu, v, 8);
    if (lane >= 8) v = fma(z8, t, v);
    t = __shfl_up_sync(0xffffffffu, v, 16);
    if (lane >= 16) v = fma(z16, t, v);
    v = fma(zl, carry, v);
    if (k < n) p[k] = v;
    carry = __shfl_sync(0xffffffffu, v, 31);
  }
  __syncwarp();
  const double tail = spline_tail(p[n - 1], s_end6);
  carry = 0.0;
  for (int b = 0; b < n; b += 32) {
    const int k = n - 1 - (b + lane);   // lane 0 of the first chunk is the last element
    double v = k >= 0 ? -z * p[k] : 0.0;
    if (k == n - 1) v = tail;
    double t = __shfl_up_sync(0xffffffffu, v, 1);
    if (lane >= 1) v = fma(z, t, v);
    t = __shfl_up_sync(0xffffffffu, v, 2);
    if (lane >= 2) v = fma(z2, t, v);
    t = __shfl_up_sync(0xffffffffu, v, 4);
    if (lane >= 4) v = fma(z4, t, v);
    t = __shfl_up_sync(0xffffffffu, v, 8);
    if (lane >= 8) v = fma(z8, t, v);
    t = __shfl_up_sync(0xffffffffu, v, 16);
    if (lane >= 16) v = fma(z16, t, v);
    v = fma(zl, carry, v);
    if (k >= 0) p[k] = v;
    carry = __shfl_sync(0xffffffffu, v, 31);
  }
}

// Strided lines (y or z), split into segments of kSplineSeg elements, one
// thread per (line, segment), consecutive threads on consecutive lines.  A
// segment's recursion starts kSplineWarm elements early from zero (its error
// decays as |z|^28 < 1e-16) unless that reaches the line's end, where the
// exact start value is used.  Out of place: the causal pass reads src and
// writes c+ to dst, storing c-[n-1] in place of c+[n-1]; the anti-causal
// pass reads that and writes c- back.  Line i starts at
// (i % na) * sa + (i / na) * sb, elements `stride` apart.
constexpr int kSplineSeg = 64, kSplineWarm = 28;

__global__ void k_spline_causal(const double* __restrict__ src, double* __restrict__ dst, long long nlines, int n,
                                long long stride, long long na, long long sa, long long sb) {
  const double z = kSplineZ;
  const int nseg = (n + kSplineSeg - 1) / kSplineSeg;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= nlines * nseg) return;
  const long long line = i % nlines;
  const int sgm = (int)(i / nlines);
  const long long base = (line % na) * sa + (line / na) * sb;
  const int k0 = sgm * kSplineSeg, k1 = min(k0 + kSplineSeg, n), kw = max(k0 - kSplineWarm, 0);
  double c;
  int k;
  if (kw == 0) {
    c = 6.0 * src[base] / (1.0 - z);
    if (k0 == 0) dst[base] = c;
    k = 1;
  } else {
    c = 0.0;
    k = kw;
  }
  for (; k < k1; ++k) {
    c = fma(z, c, 6.0 * src[base + k * stride]);
    if (k >= k0) dst[base + k * stride] = c;
  }
  if (k1 == n) dst[base + (long long)(n - 1) * stride] = spline_tail(c, 6.0 * src[base + (long long)(n - 1) * stride]);
}

__global__ void k_spline_anticausal(const double* __restrict__ src, double* __restrict__ dst, long long nlines, int n,
                                    long long stride, long long na, long long sa, long long sb) {
  const double z = kSplineZ;
  const int nseg = (n + kSplineSeg - 1) / kSplineSeg;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= nlines * nseg) return;
  const long long line = i % nlines;
  const int sgm = (int)(i / nlines);
  const long long base = (line % na) * sa + (line / na) * sb;
  const int k0 = sgm * kSplineSeg, k1 = min(k0 + kSplineSeg, n), ke = min(k1 + kSplineWarm, n);
  double c;
  int k;
  if (ke == n) {
    c = src[base + (long long)(n - 1) * stride];
    if (n - 1 < k1) dst[base + (long long)(n - 1) * stride] = c;
    k = n - 2;
  } else {
    c = 0.0;
    k = ke - 1;
  }
  for (; k >= k0; --k) {
    c = z * (c - src[base + k * stride]);
    if (k < k1) dst[base + k * stride] = c;
  }
}

// exclusion bit of a (resized) mask: bit 0 = (value > thresh)
template <typename T>
__global__ void k_threshold_bits(const T* __restrict__ in, uint8_t* __restrict__ bits, long long n, double thresh) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    bits[i] = (double)in[i] > thresh ? 1 : 0;
}

// One axis of a spline sample: the padded coordinate c + 12, clamped to the
// padded extent [0, np - 1] like mode "nearest" does, split into the first of
// the four taps and the fraction.  The clamp is applied to c itself, so the
// fraction carries no rounding from the shift.
struct SplineAxis {
  int i[4];
  float t;
};

__device__ __forceinline__ SplineAxis spline_axis(float c, int np) {
  const float lo = -(float)kSplinePad, hi = (float)(np - 1 - kSplinePad);
  if (!(c >= lo)) c = lo;
  if (!(c <= hi)) c = hi;
  const float f = floorf(c);
  SplineAxis a;
  a.t = c - f;
  const int i0 = (int)f + kSplinePad - 1;
#pragma unroll
  for (int k = 0; k < 4; ++k) a.i[k] = clampi(i0 + k, 0, np - 1);
  return a;
}

template <typename R>
__device__ __forceinline__ void bspline_weights(R t, R w[4]) {
  const R t2 = t * t, t3 = t2 * t, u = R(1) - t;
  w[0] = u * u * u / R(6);
  w[1] = (R(3) * t3 - R(6) * t2 + R(4)) / R(6);
  w[2] = (-R(3) * t3 + R(3) * t2 + R(3) * t + R(1)) / R(6);
  w[3] = t3 / R(6);
}

// Cubic B-spline value of padded coefficients C (px, py, pz) at (x, y, z) in
// the unpadded index space, accumulated in R.
template <typename R, typename T>
__device__ __forceinline__ R spline_sample(const T* __restrict__ C, int px, int py, int pz, float x, float y, float z) {
  const SplineAxis ax = spline_axis(x, px), ay = spline_axis(y, py), az = spline_axis(z, pz);
  R wx[4], wy[4], wz[4];
  bspline_weights<R>((R)ax.t, wx);
  bspline_weights<R>((R)ay.t, wy);
  bspline_weights<R>((R)az.t, wz);
  R acc = 0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    R accy = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const T* row = C + ((size_t)az.i[c] * py + ay.i[b]) * px;
      const R s = wx[0] * (R)__ldg(row + ax.i[0]) + wx[1] * (R)__ldg(row + ax.i[1]) + wx[2] * (R)__ldg(row + ax.i[2]) +
                  wx[3] * (R)__ldg(row + ax.i[3]);
      accy += wy[b] * s;
    }
    acc += wz[c] * accy;
  }
  return acc;
}

// Brick bounds of a mask's spline coefficients: for each 4x4x4 brick b of
// the padded volume, (min, max) of the coefficients over [4b, 4b + 6] per
// axis (the brick and the next one), rounded outward to float.  A sample
// whose first taps (spline_axis .i[0]) fall in brick b reads only
// coefficients in that range, and its value is a convex combination of them
// (the cubic B-spline weights are non-negative and sum to 1): when the
// range lies below 0.5 - 1e-4 the sample is not above 0.5, when it lies above
// 0.5 + 1e-4 it is, whatever the rounding of the 64-tap sum (its error is
// below 1e-14 of the largest coefficient).
constexpr int kBrick = 4;
constexpr float kBoundMargin = 1e-4f;

__host__ __device__ inline int brick_count(int np) { return (np + kBrick - 1) / kBrick; }

// stage 1: exact min / max of each brick, rounded outward
__global__ void k_brick_minmax(const double* __restrict__ C, int px, int py, int pz, float2* __restrict__ out) {
  const int nbx = brick_count(px), nby = brick_count(py), nbz = brick_count(pz);
  const long long nb = (long long)nbx * nby * nbz;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nb; b += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(b % nbx);
    const long long rest = b / nbx;
    const int by = (int)(rest % nby), bz = (int)(rest / nby);
    double lo = INFINITY, hi = -INFINITY;
    for (int z = bz * kBrick; z < min(pz, bz * kBrick + kBrick); ++z)
      for (int y = by * kBrick; y < min(py, by * kBrick + kBrick); ++y) {
        const double* row = C + ((size_t)z * py + y) * px;
        for (int x = bx * kBrick; x < min(px, bx * kBrick + kBrick); ++x) {
          const double v = row[x];
          lo = fmin(lo, v);
          hi = fmax(hi, v);
        }
      }
    out[b] = make_float2(__double2float_rd(lo), __double2float_ru(hi));
  }
}

// stage 2: each brick's range joined with its successors' along x, y and z
__global__ void k_brick_dilate(const float2* __restrict__ in, int px, int py, int pz, float2* __restrict__ out) {
  const int nbx = brick_count(px), nby = brick_count(py), nbz = brick_count(pz);
  const long long nb = (long long)nbx * nby * nbz;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nb; b += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(b % nbx);
    const long long rest = b / nbx;
    const int by = (int)(rest % nby), bz = (int)(rest / nby);
    float lo = INFINITY, hi = -INFINITY;
    for (int z = bz; z <= min(bz + 1, nbz - 1); ++z)
      for (int y = by; y <= min(by + 1, nby - 1); ++y)
        for (int x = bx; x <= min(bx + 1, nbx - 1); ++x) {
          const float2 v = in[((size_t)z * nby + y) * nbx + x];
          lo = fminf(lo, v.x);
          hi = fmaxf(hi, v.y);
        }
    out[b] = make_float2(lo, hi);
  }
}

// H_mask(x, y, z) > 0.5 evaluated as (float)spline_sample<double> > 0.5f,
// decided from the brick bounds wherever they settle it
__device__ __forceinline__ bool mask_above_half(const double* __restrict__ C, const float2* __restrict__ bounds, int px,
                                                int py, int pz, float x, float y, float z) {
  if (bounds) {
    const int bx = spline_axis(x, px).i[0] / kBrick, by = spline_axis(y, py).i[0] / kBrick;
    const int bz = spline_axis(z, pz).i[0] / kBrick;
    const float2 b = __ldg(bounds + ((size_t)bz * brick_count(py) + by) * brick_count(px) + bx);
    if (b.y < 0.5f - kBoundMargin) return false;
    if (b.x > 0.5f + kBoundMargin) return true;
  }
  return (float)spline_sample<double, double>(C, px, py, pz, x, y, z) > 0.5f;
}

// The float32 coefficients of a level stored as x quads: Q[row][q] holds the
// four taps (q - 1 .. q + 2, clamped to the row) a sample whose first x tap
// is q - 1 reads, so one 16-byte load replaces four scalar loads.
__global__ void k_spline_quads(const double* __restrict__ c, float4* __restrict__ q, int px, long long rows) {
  const long long n = rows * px;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % px);
    const double* r = c + (i - x);
    q[i] = make_float4((float)r[max(x - 1, 0)], (float)r[x], (float)r[min(x + 1, px - 1)], (float)r[min(x + 2, px - 1)]);
  }
}

// spline_sample<float, float> on the quad layout
__device__ __forceinline__ float spline_sample_quads(const float4* __restrict__ Q, int px, int py, int pz, float x,
                                                     float y, float z) {
  const SplineAxis ay = spline_axis(y, py), az = spline_axis(z, pz);
  float c = x;
  const float lo = -(float)kSplinePad, hi = (float)(px - 1 - kSplinePad);
  if (!(c >= lo)) c = lo;
  if (!(c <= hi)) c = hi;
  const float f = floorf(c);
  const int qx = (int)f + kSplinePad;   // first tap + 1, in [0, px - 1]
  float wx[4], wy[4], wz[4];
  bspline_weights<float>(c - f, wx);
  bspline_weights<float>(ay.t, wy);
  bspline_weights<float>(az.t, wz);
  float acc = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float accy = 0.f;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const float4 v = __ldg(Q + ((size_t)az.i[k] * py + ay.i[b]) * px + qx);
      accy += wy[b] * (wx[0] * v.x + wx[1] * v.y + wx[2] * v.z + wx[3] * v.w);
    }
    acc += wz[k] * accy;
  }
  return acc;
}

// ---------------------------------------------------------------------------
// fused iteration
// ---------------------------------------------------------------------------

struct XresArgs {
  IterArgs a;              // iteration grid: a.ref = moving level, a.mbits bit 0 = moving exclusion
  const float4* g;         // reference level on its grid: (m, Gx, Gy, Gz), G = half central difference
  int nxh, nyh, nzh;       // reference level extent
  const float4* cref;      // padded spline coefficients of the reference level, x quads
  const double* cmask;     // padded spline coefficients of its 0/1 exclusion mask, or null
  const float2* cbounds;   // their brick bounds (mask_above_half), or null
  int pxh, pyh, pzh;       // padded extent
  double zr, zrh;          // zRatio / 2^l and zRatio_HR / 2^l: phase z of slice k is k zr / zrh
  const float4* phase0;    // the level's initial phase (x, y, z, -), or null for (x, y, z zr / zrh)
  float* it_out;           // non-null: every voxel's It_raw (mov - H(phase)) is stored here,
  uint8_t* ex_out;         //   and its exclusion flag here (the end-of-pass evaluation)
};

// One launch of the cross-resolution iteration: per voxel the residual
// mov - H(phase) with phase = (x, y, z zr / zrh) + motion, the reference's
// gradient at the phase, exclusion by the moving mask or H_mask(phase) > 0.5,
// then the same smoothing, window sums and CP neighbour difference as
// k_lk_accumulate (utils/calFlowCrossResolution.py:2101-2170).  Four CTAs
// per SM (64 registers, some spills to L1): the kernel waits on the latency
// of its spline gathers, and the fourth CTA hides more of it than the spills
// cost (32.4 -> 29.8 ms per 32x1024x1024 registration against three CTAs).
template <int MODE, int DIFF0, bool MASK>
__global__ void __launch_bounds__(kAccThreads, 4) k_xres_accumulate(const __grid_constant__ XresArgs xa) {
  const IterArgs& a = xa.a;
  if (!*(volatile const int*)&a.st->active) return;
  extern __shared__ float4 smem4[];
  const int nx = a.mov.nx, ny = a.mov.ny, nz = a.mov.nz;
  const int w = a.w;
  const int ncx = a.cpv.ncx, ncy = a.cpv.ncy;
  const AccSmem sm(smem4, w);
  float4* gsm = sm.gsm;
  float* it_raw = sm.it_raw;
  const TileField tf = sm.tf;
  int* flags = sm.flags;
  float* red = sm.red;
  const TileField tf0 = sm.tf0;
  int* flags0 = sm.flags0;
  float dmax = 0.f;
  const int ntiles = nz * a.ntx * a.nty;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
#include "wr_xres_tile.inc"
  }
  if (DIFF0 != kNoDiff) {
    const float mx = block_max(dmax, red);
    if (threadIdx.x == 0 && mx > 0.f) atomicMax(&a.st->maxdiff_bits, __float_as_uint(mx));
  }
}

// (n, 3) interleaved float -> float4 (the finest level's initial phase: an
// exact copy, as a resize at scale 1 is)
__global__ void k_pack_xyz(const float* __restrict__ in, float4* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = make_float4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0.f);
}

// Final outputs at the finest level: phase = (x, y, z zr / zrh) + motion,
// the motion itself and H(phase) (utils/calFlowCrossResolution.py:2205-2209).
template <int MODE>
__global__ void k_xres_finish(const FieldSrc f, float* __restrict__ phase, float* __restrict__ motion,
                              float* __restrict__ sampled, const float4* __restrict__ cref, int pxh, int pyh, int pzh,
                              int nx, int ny, int nz, double zr, double zrh, const float4* __restrict__ phase0) {
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    const float fz0 = (float)(((double)z * zr) / zrh);
    WR_FOR_COLS(nx, x) {
      const float3 m = eval_field<MODE>(f, x, y, z);
      const size_t i = ((size_t)z * ny + y) * nx + x;
      float px = (float)x + m.x, py = (float)y + m.y, pz = fz0 + m.z;
      if (phase0) {
        const float4 q = phase0[i];
        px = q.x + m.x;
        py = q.y + m.y;
        pz = q.z + m.z;
      }
      if (motion) {
        motion[3 * i] = m.x;
        motion[3 * i + 1] = m.y;
        motion[3 * i + 2] = m.z;
      }
      if (phase) {
        phase[3 * i] = px;
        phase[3 * i + 1] = py;
        phase[3 * i + 2] = pz;
      }
      if (sampled) sampled[i] = spline_sample_quads(cref, pxh, pyh, pzh, px, py, pz);
    }
  }
}

// ---------------------------------------------------------------------------
// continuous reference H (generate_continuous_H_gpu / apply_H_to_matrix_gpu,
// utils/calFlowCrossResolution.py:463-478, 1144-1154) and the fixed-plane
// projections of mapped samples (:480-660, 700-1141)
// ---------------------------------------------------------------------------

// H at n points (x, y, z) of `coords`: float64 coefficients, float64 sum,
// rounded to float32 like map_coordinates on a float32 stack.
__global__ void k_spline_points(const double* __restrict__ C, int px, int py, int pz, const float* __restrict__ coords,
                                long long n, float* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)spline_sample<double, double>(C, px, py, pz, coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);
}

// float <-> unsigned key whose unsigned order is the float order
__device__ __forceinline__ unsigned float_key(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// minimum of the finite values (key in mm[0], start 0xffffffff) and whether
// there is one (mm[1] != 0)
__global__ void k_finite_min(const float* __restrict__ v, long long n, unsigned* __restrict__ mm) {
  unsigned kmin = 0xffffffffu, any = 0u;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float f = v[i];
    if (isfinite(f)) {
      kmin = min(kmin, float_key(f));
      any = 1u;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
    any |= __shfl_xor_sync(0xffffffffu, any, o);
  }
  if ((threadIdx.x & 31) == 0 && any) {
    atomicMin(mm, kmin);
    atomicOr(mm + 1, 1u);
  }
}

// shift = max(1 - min, 0) of the finite values, as a float32 computation
__device__ __forceinline__ float project_shift(const unsigned* mm) {
  if (!mm[1]) return 0.f;
  return fmaxf(__fadd_rn(-key_float(mm[0]), 1.f), 0.f);
}

// Max splat of shifted (non-negative) samples onto fixed z planes: a sample
// at (x, y, z) reaches plane z0 when |z - z0| <= z_window and writes the XY
// pixels (rounded x, y) or (floor .. floor + 1 +- extra), each pixel index
// divided by the down-sampling factor.  Output (nplanes, xout, yout) as
// unsigned keys, start 0 (below every float).
__global__ void k_project_max(const float* __restrict__ values, const float* __restrict__ coords, long long n,
                              const float* __restrict__ target_z, int nplanes, int xref, int yref, int xout, int yout,
                              float z_window, int ds, int nearest, int extra, const unsigned* __restrict__ mm,
                              unsigned* __restrict__ out) {
  const float shift = project_shift(mm);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float v0 = values[i];
    const float x = coords[3 * i], y = coords[3 * i + 1], z = coords[3 * i + 2];
    const float val = __fadd_rn(v0, shift);
    if (!isfinite(val) || !isfinite(x) || !isfinite(y) || !isfinite(z)) continue;
    const unsigned key = float_key(val);
    int x0, x1, y0, y1;
    if (nearest) {
      x0 = x1 = (int)floorf(x + 0.5f);
      y0 = y1 = (int)floorf(y + 0.5f);
    } else {
      const int xf = (int)floorf(x), yf = (int)floorf(y);
      x0 = xf - extra; x1 = xf + 1 + extra;
      y0 = yf - extra; y1 = yf + 1 + extra;
    }
    for (int p = 0; p < nplanes; ++p) {
      if (fabsf(z - target_z[p]) > z_window) continue;
      unsigned* plane = out + (size_t)p * xout * yout;
      for (int xi = max(x0, 0); xi <= min(x1, xref - 1); ++xi) {
        const int xo = xi / ds;
        if (xo >= xout) continue;
        for (int yi = max(y0, 0); yi <= min(y1, yref - 1); ++yi) {
          const int yo = yi / ds;
          if (yo >= yout) continue;
          atomicMax(plane + (size_t)xo * yout + yo, key);
        }
      }
    }
  }
}

// keys -> values: the max minus the shift, or the fill value where nothing
// landed (has_fill = 0 keeps -inf)
__global__ void k_project_max_finish(const unsigned* __restrict__ keys, long long n, const unsigned* __restrict__ mm,
                                     float fill, int has_fill, float* __restrict__ out) {
  const float shift = project_shift(mm);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned k = keys[i];
    if (k == 0u) out[i] = has_fill ? fill : -INFINITY;
    else out[i] = __fsub_rn(key_float(k), shift);
  }
}

// Weighted splat: samples with x in [0, xref - 1] and y in [0, yref - 1]
// reach plane z0 with weight wz(|z - z0|) (mode 0: 1, 1: 1 - dz / (window +
// 1e-6), 2: exp(-dz^2 / (2 sigma^2 + 1e-6))) for dz <= z_window, and are
// spread bilinearly over the 2 x 2 output pixels around (x, y) / ds.
__global__ void k_project_weighted(const float* __restrict__ values, const float* __restrict__ coords, long long n,
                                   const float* __restrict__ target_z, int nplanes, int xref, int yref, int xout,
                                   int yout, float z_window, float z_sigma, int ds, int mode, float* __restrict__ sum_v,
                                   float* __restrict__ sum_w) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float v = values[i];
    const float x = coords[3 * i], y = coords[3 * i + 1], z = coords[3 * i + 2];
    if (!isfinite(v) || !isfinite(x) || !isfinite(y) || !isfinite(z)) continue;
    if (x < 0.f || x > (float)(xref - 1) || y < 0.f || y > (float)(yref - 1)) continue;
    const float xo_f = x / (float)ds, yo_f = y / (float)ds;
    const int xo0 = (int)floorf(xo_f), yo0 = (int)floorf(yo_f);
    const float dx = xo_f - (float)xo0, dy = yo_f - (float)yo0;
    for (int p = 0; p < nplanes; ++p) {
      const float dz = fabsf(z - target_z[p]);
      if (dz > z_window) continue;
      float wz = 1.f;
      if (mode == 1) {
        wz = fmaxf(1.f - dz / (z_window + 1e-6f), 0.f);
      } else if (mode == 2) {
        const float sg = z_sigma > 0.f ? z_sigma : z_window * 0.5f;
        wz = expf(-0.5f * dz * dz / (sg * sg + 1e-6f));
      }
      if (!(wz > 0.f) || !isfinite(wz)) continue;
      const size_t base = (size_t)p * xout * yout;
      for (int ax = 0; ax <= 1; ++ax) {
        const int xo = xo0 + ax;
        if (xo < 0 || xo >= xout) continue;
        const float wx = ax == 0 ? 1.f - dx : dx;
        for (int ay = 0; ay <= 1; ++ay) {
          const int yo = yo0 + ay;
          if (yo < 0 || yo >= yout) continue;
          const float w = wx * (ay == 0 ? 1.f - dy : dy) * wz;
          if (!(w > 0.f) || !isfinite(w)) continue;
          atomicAdd(sum_v + base + (size_t)xo * yout + yo, v * w);
          atomicAdd(sum_w + base + (size_t)xo * yout + yo, w);
        }
      }
    }
  }
}

__global__ void k_project_weighted_finish(const float* __restrict__ sum_v, const float* __restrict__ sum_w, long long n,
                                          float eps, float fill, float* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float w = sum_w[i];
    out[i] = w > eps ? sum_v[i] / fmaxf(w, eps) : fill;
  }
}

}  // namespace wr
