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

__global__ void k_f64_to_f32(const double* __restrict__ in, float* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
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

// ---------------------------------------------------------------------------
// fused iteration
// ---------------------------------------------------------------------------

struct XresArgs {
  IterArgs a;              // iteration grid: a.ref = moving level, a.mbits bit 0 = moving exclusion
  const float4* g;         // reference level on its grid: (m, Gx, Gy, Gz), G = half central difference
  int nxh, nyh, nzh;       // reference level extent
  const float* cref;       // padded spline coefficients of the reference level
  const double* cmask;     // padded spline coefficients of its 0/1 exclusion mask, or null
  int pxh, pyh, pzh;       // padded extent
  double zr, zrh;          // zRatio / 2^l and zRatio_HR / 2^l: phase z of slice k is k zr / zrh
};

// One launch of the cross-resolution iteration: per voxel the residual
// mov - H(phase) with phase = (x, y, z zr / zrh) + motion, the reference's
// gradient at the phase, exclusion by the moving mask or H_mask(phase) > 0.5,
// then the same smoothing, window sums and CP neighbour difference as
// k_lk_accumulate (utils/calFlowCrossResolution.py:2101-2170).
template <int MODE, int DIFF0, bool MASK>
__global__ void __launch_bounds__(kAccThreads, 2) k_xres_accumulate(const __grid_constant__ XresArgs xa) {
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

// Final outputs at the finest level: phase = (x, y, z zr / zrh) + motion,
// the motion itself and H(phase) (utils/calFlowCrossResolution.py:2205-2209).
template <int MODE>
__global__ void k_xres_finish(const FieldSrc f, float* __restrict__ phase, float* __restrict__ motion,
                              float* __restrict__ sampled, const float* __restrict__ cref, int pxh, int pyh, int pzh,
                              int nx, int ny, int nz, double zr, double zrh) {
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    const float fz0 = (float)(((double)z * zr) / zrh);
    WR_FOR_COLS(nx, x) {
      const float3 m = eval_field<MODE>(f, x, y, z);
      const size_t i = ((size_t)z * ny + y) * nx + x;
      const float px = (float)x + m.x, py = (float)y + m.y, pz = fz0 + m.z;
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
      if (sampled) sampled[i] = spline_sample<float, float>(cref, pxh, pyh, pzh, px, py, pz);
    }
  }
}

}  // namespace wr
