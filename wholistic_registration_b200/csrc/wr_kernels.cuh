// Device kernels of the pyramid patch-wise Lucas-Kanade registration path.
//
// Layout: every volume is C-contiguous (z, y, x), x fastest.  A level's moving
// volume is stored as float4 (m, Gx, Gy, Gz): the value and its clamped
// central differences, so that the warp sample and the three gradient samples
// of utils/calFlow3d_Wei_v1.py:134-206 come out of one set of 8 corner loads
// (see lk_accumulate).  Control points (CP) are float4 (dx, dy, dz, 0).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "wr_plan.h"
#include "wr_resize_table.cuh"

namespace wr {

constexpr int kThreads = 256;

// ---------------------------------------------------------------------------
// element loads
// ---------------------------------------------------------------------------

template <typename T> __device__ __forceinline__ float load_f(const T* p, size_t i);
template <> __device__ __forceinline__ float load_f<uint16_t>(const uint16_t* p, size_t i) {
  return (float)__ldg(p + i);
}
template <> __device__ __forceinline__ float load_f<uint8_t>(const uint8_t* p, size_t i) {
  return (float)__ldg(p + i);
}
template <> __device__ __forceinline__ float load_f<float>(const float* p, size_t i) {
  return __ldg(p + i);
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Row-parallel voxel loops: blocks of 32 x kRowWarps threads; warp
// threadIdx.y of a block takes rows in turn and its lanes take the columns,
// so that voxel kernels need no per-voxel integer division.
constexpr int kRowWarps = 8;
#define WR_FOR_ROWS(nrows, wr_row_) \
  for (int wr_row_ = blockIdx.x * kRowWarps + threadIdx.y; wr_row_ < (nrows); wr_row_ += gridDim.x * kRowWarps)
#define WR_FOR_COLS(ncols, wr_col_) for (int wr_col_ = threadIdx.x; wr_col_ < (ncols); wr_col_ += 32)

// f32 coordinate -> (lower tap, fraction); huge values are pinned so the
// integer conversion stays defined (the taps are clamped anyway).
__device__ __forceinline__ void split_coord(float c, int& i0, float& t) {
  c = fminf(fmaxf(c, -1048576.f), 1048576.f);
  float f = floorf(c);
  t = c - f;
  i0 = (int)f;
}

// Storage of a level's (m, Gx, Gy, Gz) and of the reference level.
// WR_PREC_F32: float4 / float.  WR_PREC_F16: 4 x half / half holding half
// the value (so that uint16 data, up to 65535, stays inside the float16
// range), scaled back by 2 on load.  WR_PREC_BF16: 4 x bfloat16 / bfloat16.
template <int PREC> struct Store;
template <> struct Store<WR_PREC_F32> {
  typedef float4 V4;
  typedef float V1;
  static __device__ __forceinline__ float4 load4(const V4* p) { return __ldg(p); }
  static __device__ __forceinline__ float load_m(const V4* p) { return __ldg(reinterpret_cast<const float*>(p)); }
  static __device__ __forceinline__ float load1(const V1* p) { return __ldg(p); }
  static __device__ __forceinline__ V4 pack4(float4 v) { return v; }
  static __device__ __forceinline__ V1 pack1(float v) { return v; }
};
template <> struct Store<WR_PREC_F16> {
  typedef uint2 V4;
  typedef __half V1;
  static __device__ __forceinline__ float4 load4(const V4* p) {
    const uint2 u = __ldg(p);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
    return make_float4(2.f * a.x, 2.f * a.y, 2.f * b.x, 2.f * b.y);
  }
  static __device__ __forceinline__ float load_m(const V4* p) {
    return 2.f * __half2float(__ldg(reinterpret_cast<const __half*>(p)));
  }
  static __device__ __forceinline__ float load1(const V1* p) { return 2.f * __half2float(__ldg(p)); }
  static __device__ __forceinline__ V4 pack4(float4 v) {
    __half2 a = __floats2half2_rn(0.5f * v.x, 0.5f * v.y), b = __floats2half2_rn(0.5f * v.z, 0.5f * v.w);
    return make_uint2(*reinterpret_cast<unsigned*>(&a), *reinterpret_cast<unsigned*>(&b));
  }
  static __device__ __forceinline__ V1 pack1(float v) { return __float2half_rn(0.5f * v); }
};
template <> struct Store<WR_PREC_BF16> {
  typedef uint2 V4;
  typedef __nv_bfloat16 V1;
  static __device__ __forceinline__ float4 load4(const V4* p) {
    const uint2 u = __ldg(p);
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
    const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
    return make_float4(a.x, a.y, b.x, b.y);
  }
  static __device__ __forceinline__ float load_m(const V4* p) {
    return __bfloat162float(__ldg(reinterpret_cast<const __nv_bfloat16*>(p)));
  }
  static __device__ __forceinline__ float load1(const V1* p) { return __bfloat162float(__ldg(p)); }
  static __device__ __forceinline__ V4 pack4(float4 v) {
    __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
    return make_uint2(*reinterpret_cast<unsigned*>(&a), *reinterpret_cast<unsigned*>(&b));
  }
  static __device__ __forceinline__ V1 pack1(float v) { return __float2bfloat16_rn(v); }
};

// float16 storage holds half of each value: a half2 result as float2, doubled
__device__ __forceinline__ float2 half2_scaled(__half2 h) {
  const float2 f = __half22float2(h);
  return make_float2(2.f * f.x, 2.f * f.y);
}

// ---------------------------------------------------------------------------
// resize tables (utils/imresize.py:60-82)
// ---------------------------------------------------------------------------

// One thread per output row: P candidate taps, float64, unmodified order.
__global__ void k_build_table(double* w, int32_t* idx, int in_len, int out_len, int method, int P) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= out_len) return;
  resize_row(in_len, out_len, method, k, w + (size_t)k * P, idx + (size_t)k * P);
}

// [n][P] -> [P][n]: in the x pass the lanes of a warp hold consecutive
// outputs and then read consecutive weights and indexes.
__global__ void k_transpose_table(const double* __restrict__ w, const int32_t* __restrict__ idx, double* wt,
                                  int32_t* it, int n, int P) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)n * P) return;
  const int k = (int)(i / P), t = (int)(i - (long long)k * P);
  wt[(size_t)t * n + k] = w[i];
  it[(size_t)t * n + k] = idx[i];
}

// Bilinear up-sampling table compacted to the (at most two) taps with nonzero
// weight.  Dropping exact-zero terms does not change the weighted sum.
__global__ void k_build_up_table(float* w2, int32_t* i2, int in_len, int out_len, int* err_flag) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= out_len) return;
  double w[16];
  int32_t ix[16];
  int P = resize_taps(in_len, out_len);
  if (P > 16) { atomicOr(err_flag, 1); return; }
  resize_row(in_len, out_len, RESIZE_BILINEAR, k, w, ix);
  int n = 0;
  float ow[2] = {0.f, 0.f};
  int32_t oi[2] = {0, 0};
  for (int t = 0; t < P; ++t) {
    if (w[t] != 0.0) {
      if (n < 2) { ow[n] = (float)w[t]; oi[n] = ix[t]; }
      ++n;
    }
  }
  if (n > 2) atomicOr(err_flag, 2);
  w2[2 * k] = ow[0]; w2[2 * k + 1] = ow[1];
  i2[2 * k] = oi[0]; i2[2 * k + 1] = oi[1];
}

// ---------------------------------------------------------------------------
// separable resample (utils/imresize.py:121-137, 185-187)
// ---------------------------------------------------------------------------

// Float64 accumulation without contraction reproduces the reference's
// float64 products and tap-order sums exactly; float32 uses FMA with the
// weight rounded to float32.
template <typename A> struct Acc;
template <> struct Acc<double> {
  static __device__ __forceinline__ double madd(double acc, double w, double v) {
    return __dadd_rn(acc, __dmul_rn(w, v));
  }
  static __device__ __forceinline__ double si_weight(const SITaps& si, int t) { return si.w[t]; }
};
template <> struct Acc<float> {
  static __device__ __forceinline__ float madd(float acc, double w, float v) {
    return fmaf((float)w, v, acc);
  }
  static __device__ __forceinline__ float madd(float acc, float w, float v) { return fmaf(w, v, acc); }
  static __device__ __forceinline__ float si_weight(const SITaps& si, int t) { return si.wf[t]; }
};

// Separable resize passes.  Outputs inside the table's shift-invariant
// interior (SITaps) read their taps at s*o + c0 + t with the weights held in
// the kernel parameters; the few outputs near the edges (reflected taps) read
// the table, x tables tap-major ([tap][output]), y tables output-major.
// stride/comp select one component of an interleaved input.

// out[z][y][xo] = sum_t w[t][xo] * in[z][y][idx[t][xo]]
template <typename Tin, typename A, typename Tout>
__global__ void k_resample_x(const __grid_constant__ SITaps si, const Tin* __restrict__ in, Tout* __restrict__ out,
                             int nz, int ny, int nx_in, int nx_out, const double* __restrict__ w,
                             const int32_t* __restrict__ idx, int P, int stride, int comp) {
  WR_FOR_ROWS(nz * ny, row) {
    const Tin* src = in + (size_t)row * nx_in * stride + comp;
    Tout* dst = out + (size_t)row * nx_out;
    WR_FOR_COLS(nx_out, xo) {
      A acc = 0;
      if (xo >= si.lo && xo < si.hi) {
        const Tin* q = src + (size_t)(si.s * xo + si.c0) * stride;
#pragma unroll 4
        for (int t = 0; t < si.P; ++t) acc = Acc<A>::madd(acc, Acc<A>::si_weight(si, t), (A)__ldg(q + (size_t)t * stride));
      } else {
        for (int t = 0; t < P; ++t)
          acc = Acc<A>::madd(acc, __ldg(w + (size_t)t * nx_out + xo),
                             (A)__ldg(src + (size_t)__ldg(idx + (size_t)t * nx_out + xo) * stride));
      }
      dst[xo] = (Tout)acc;
    }
  }
}

// The x pass with each row staged in shared memory, for an integer down-scale
// factor S (P = 4S + 2 candidate taps, fixed at compile time): one warp per
// row; the row is read once with coalesced loads and stored in polyphase
// order, so interior outputs read their taps from shared memory without bank
// conflicts and with the weights as constant operands; edge outputs read the
// table.  Blocks of 32 x kStageWarps threads; dynamic shared memory
// kStageWarps * S * ls elements of A.
constexpr int kStageWarps = 4;
template <int S, typename Tin, typename A, typename Tout>
__global__ void __launch_bounds__(32 * kStageWarps) k_resample_x_si(
    const __grid_constant__ SITaps si, const Tin* __restrict__ in, Tout* __restrict__ out, int nrows, int nx_in,
    int nx_out, const double* __restrict__ w, const int32_t* __restrict__ idx) {
  constexpr int NP = 4 * S + 2;
  extern __shared__ __align__(16) unsigned char stage_raw[];
  const int ls = si.ls;
  A* buf = reinterpret_cast<A*>(stage_raw) + (size_t)threadIdx.y * S * ls;
  const int lane = threadIdx.x;
  for (int row = blockIdx.x * kStageWarps + threadIdx.y; row < nrows; row += gridDim.x * kStageWarps) {
    const Tin* src = in + (size_t)row * nx_in;
    for (int e0 = 0; e0 < nx_in; e0 += 32 * 8) {
      A v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int e = e0 + 32 * k + lane;
        v[k] = e < nx_in ? (A)__ldg(src + e) : (A)0;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int e = e0 + 32 * k + lane;
        if (e < nx_in) buf[(e % S) * ls + e / S] = v[k];
      }
    }
    __syncwarp();
    Tout* dst = out + (size_t)row * nx_out;
    for (int xo = lane; xo < nx_out; xo += 32) {
      A acc = 0;
      if (xo >= si.lo && xo < si.hi) {
#pragma unroll
        for (int t = 0; t < NP; ++t) acc = Acc<A>::madd(acc, Acc<A>::si_weight(si, t), buf[si.off[t] + xo]);
      } else {
        for (int t = 0; t < NP; ++t)
          acc = Acc<A>::madd(acc, __ldg(w + (size_t)t * nx_out + xo), (A)__ldg(src + __ldg(idx + (size_t)t * nx_out + xo)));
      }
      dst[xo] = (Tout)acc;
    }
    __syncwarp();
  }
}

// First tap of an interior output of the antialiased bicubic table for an
// integer down-scale factor S: taps s * o + kPPFirstTap<S> + t, t < 4S + 2
// (utils/imresize.py:60-82 with width 4S; the host checks the table against it).
template <int S> constexpr int kPPFirstTap = -(3 * S / 2) - 1;
constexpr int kPPMaxIn = 1024;   // longest row of k_resample_x_pp
constexpr int kPPMaxEdge = 16;   // most edge outputs of a k_resample_x_pp row

// S consecutive inputs as one vector load (the row start and S * sizeof(T)
// are multiples of the vector size).
template <typename T, int S>
__device__ __forceinline__ void load_group(const T* __restrict__ p, T (&v)[S]) {
  constexpr int B = (int)sizeof(T) * S;
  if constexpr (B % 16 == 0) {
#pragma unroll
    for (int c = 0; c < B / 16; ++c) {
      const int4 q = __ldg(reinterpret_cast<const int4*>(p) + c);
      memcpy(&v[c * (16 / (int)sizeof(T))], &q, 16);
    }
  } else if constexpr (B == 8) {
    const uint2 q = __ldg(reinterpret_cast<const uint2*>(p));
    memcpy(v, &q, 8);
  } else if constexpr (B == 4) {
    const unsigned q = __ldg(reinterpret_cast<const unsigned*>(p));
    memcpy(v, &q, 4);
  } else {
#pragma unroll
    for (int j = 0; j < S; ++j) v[j] = __ldg(p + j);
  }
}

// The x pass with each row staged in polyphase order relative to the first
// tap: input e sits in phase (e - C0) mod S at index (e - C0) div S, phases
// LS elements apart.  A lane loads S consecutive inputs as one vector and
// stores each to its own phase at the lane's index (no bank conflicts), and
// tap t of interior output o sits at phase t mod S, index o + t div S: every
// staged address is a compile-time offset from the lane's column, so neither
// the staging nor the taps need address arithmetic.  Taps are summed in tap
// order as in k_resample_x_si, so the outputs are the same.  Rows of at most
// kPPMaxIn inputs.  The few edge outputs (reflected taps) read the staged row
// too: their weights and staged positions are tabulated in shared memory once
// per block, so no output waits on global memory after the row is staged.
template <int S, typename Tin, typename A, typename Tout>
__global__ void __launch_bounds__(32 * kStageWarps) k_resample_x_pp(
    const __grid_constant__ SITaps si, const Tin* __restrict__ in, Tout* __restrict__ out, int nrows, int nx_in,
    int nx_out, const double* __restrict__ w, const int32_t* __restrict__ idx) {
  constexpr int NP = 4 * S + 2;
  constexpr int C0 = kPPFirstTap<S>;
  constexpr int LS = kPPMaxIn / S + 2;   // covers index (kPPMaxIn - 1 - C0) div S
  __shared__ A stage[kStageWarps][S * LS];
  __shared__ A edge_w[kPPMaxEdge * NP];
  __shared__ int edge_pos[kPPMaxEdge * NP];
  // edge outputs: o < lo (k = o) and o >= hi (k = lo + o - hi); the host
  // checks that there are at most kPPMaxEdge
  const int nedge = si.lo + (nx_out - si.hi);
  for (int q = threadIdx.y * 32 + threadIdx.x; q < nedge * NP; q += 32 * kStageWarps) {
    const int k = q / NP, t = q - k * NP;
    const int o = k < si.lo ? k : si.hi + (k - si.lo);
    edge_w[q] = (A)__ldg(w + (size_t)t * nx_out + o);
    const int d = __ldg(idx + (size_t)t * nx_out + o) - C0;   // >= 0: C0 < 0 <= idx
    edge_pos[q] = (d % S) * LS + d / S;
  }
  __syncthreads();
  A* buf = stage[threadIdx.y];
  const int lane = threadIdx.x;
  const int ngroups = nx_in / S;
  for (int row = blockIdx.x * kStageWarps + threadIdx.y; row < nrows; row += gridDim.x * kStageWarps) {
    const Tin* src = in + (size_t)row * nx_in;
    // U groups per lane in flight (16 S-element vectors per warp row and step)
    constexpr int U = 16 / S;
    for (int m0 = 0; m0 < ngroups; m0 += 32 * U) {
      Tin v[U][S];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int m = m0 + 32 * u + lane;
        if (m < ngroups) load_group<Tin, S>(src + (size_t)S * m, v[u]);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int m = m0 + 32 * u + lane;
        if (m < ngroups) {
#pragma unroll
          for (int j = 0; j < S; ++j) {
            const int pj = ((j - C0) % S + S) % S;                       // phase of input S m + j
            const int qj = (j - C0 >= 0) ? (j - C0) / S : -((C0 - j + S - 1) / S);
            buf[pj * LS + m + qj] = (A)v[u][j];
          }
        }
      }
    }
    __syncwarp();
    Tout* dst = out + (size_t)row * nx_out;
    for (int xo = lane; xo < nx_out; xo += 32) {
      A acc = 0;
      if (xo >= si.lo && xo < si.hi) {
        const A* b = buf + xo;
#pragma unroll
        for (int t = 0; t < NP; ++t) acc = Acc<A>::madd(acc, Acc<A>::si_weight(si, t), b[(t % S) * LS + t / S]);
      } else {
        const int k = xo < si.lo ? xo : si.lo + (xo - si.hi);
        for (int t = 0; t < NP; ++t) acc = Acc<A>::madd(acc, edge_w[k * NP + t], buf[edge_pos[k * NP + t]]);
      }
      dst[xo] = (Tout)acc;
    }
    __syncwarp();
  }
}

// The x pass of a uint8 mask in float64, exact.  In a row holding only 0 and
// 1, a tap with 0 adds an exact zero and a tap with 1 adds its weight, so an
// output is the tap-order float64 sum of the weights of its set taps: 0 when
// none is set, si.wsum (the same sum over every tap) when all are; only
// windows that are mixed sum their taps.  Rows with other values take the
// plain product sums.  The row is staged as bytes plus ballot words and
// their prefix popcounts.  Rows whose length is a multiple of 32 (row starts
// 16-byte aligned) load each 32-input word as two 16-byte vectors in one lane
// and build its bits with per-byte compares; other rows load bytes and ballot.
// Per warp: the row bytes (rounded up to 16), then the words and prefixes
// (rounded up to 16 bytes): mask_stage_bytes; after the warps' stages, the
// edge table: mask_edge_bytes.
__host__ __device__ inline size_t mask_stage_bytes(int nx_in) {
  const size_t nwords = ((size_t)nx_in + 31) / 32;
  return ((size_t)nx_in + 15) / 16 * 16 + (8 * (nwords + 1) + 15) / 16 * 16;
}
template <int S>
constexpr size_t mask_edge_bytes() { return (size_t)kPPMaxEdge * (4 * S + 2) * (8 + 4); }

template <int S>
__global__ void __launch_bounds__(32 * kStageWarps) k_resample_x_mask(
    const __grid_constant__ SITaps si, const uint8_t* __restrict__ in, double* __restrict__ out, int nrows,
    int nx_in, int nx_out, const double* __restrict__ w, const int32_t* __restrict__ idx) {
  constexpr int NP = 4 * S + 2;
  extern __shared__ __align__(16) unsigned char stage_raw[];
  const int nwords = (nx_in + 31) / 32;
  const int row_bytes = (nx_in + 15) & ~15;
  unsigned char* base = stage_raw + (size_t)threadIdx.y * mask_stage_bytes(nx_in);
  const bool vec = (nx_in & 31) == 0 && ((uintptr_t)in & 15) == 0;
  uint8_t* bytes = base;
  unsigned* words = reinterpret_cast<unsigned*>(base + row_bytes);
  unsigned* prefix = words + nwords + 1;   // set taps before word k
  // edge outputs (o < lo: k = o; o >= hi: k = lo + o - hi) read the staged
  // bytes through a per-block table of weights and input positions when
  // there are at most kPPMaxEdge of them (after the per-warp stages)
  double* edge_w = reinterpret_cast<double*>(stage_raw + (size_t)kStageWarps * mask_stage_bytes(nx_in));
  int* edge_i = reinterpret_cast<int*>(edge_w + kPPMaxEdge * NP);
  const int nedge = si.lo + (nx_out - si.hi);
  const bool edge_tab = nedge <= kPPMaxEdge;
  if (edge_tab) {
    for (int q = threadIdx.y * 32 + threadIdx.x; q < nedge * NP; q += 32 * kStageWarps) {
      const int k = q / NP, t = q - k * NP;
      const int o = k < si.lo ? k : si.hi + (k - si.lo);
      edge_w[q] = __ldg(w + (size_t)t * nx_out + o);
      edge_i[q] = __ldg(idx + (size_t)t * nx_out + o);
    }
  }
  __syncthreads();
  const int lane = threadIdx.x;
  for (int row = blockIdx.x * kStageWarps + threadIdx.y; row < nrows; row += gridDim.x * kStageWarps) {
    const uint8_t* src = in + (size_t)row * nx_in;
    unsigned carry = 0;
    bool nonbinary = false;
    for (int k0 = 0; k0 < nwords; k0 += 32) {
      // lane j ends with word k0 + j: bit i = element (k0 + j) * 32 + i is set
      unsigned mine = 0;
      if (vec) {
        const int kw = k0 + lane;
        if (kw < nwords) {
          const uint4* p = reinterpret_cast<const uint4*>(src + 32 * (size_t)kw);
          const uint4 q0 = __ldg(p), q1 = __ldg(p + 1);
          const unsigned c[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            // bytes 0..3 of chunk j (elements 4j .. 4j + 3): nonzero flags to bits 4j .. 4j + 3
            const unsigned nz = __vcmpne4(c[j], 0u) & 0x01010101u;
            mine |= ((nz * 0x01020408u) >> 24) << (4 * j);
            nonbinary |= __vcmpgtu4(c[j], 0x01010101u) != 0u;
          }
          uint4* d = reinterpret_cast<uint4*>(bytes + 32 * kw);
          d[0] = q0;
          d[1] = q1;
        }
      } else {
        uint8_t v[32];
#pragma unroll
        for (int b = 0; b < 32; ++b) {
          const int e = (k0 + b) * 32 + lane;
          v[b] = e < nx_in ? __ldg(src + e) : (uint8_t)0;
        }
#pragma unroll
        for (int b = 0; b < 32; ++b) {
          const int e = (k0 + b) * 32 + lane;
          if (e < nx_in) bytes[e] = v[b];
          nonbinary |= v[b] > 1;
          const unsigned wv = __ballot_sync(0xffffffffu, v[b] != 0);
          if (lane == b) mine = wv;
        }
      }
      const int k = k0 + lane;
      const unsigned c = __popc(mine);
      unsigned incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned n = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += n;
      }
      if (k < nwords) {
        words[k] = mine;
        prefix[k] = carry + incl - c;
      }
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) prefix[nwords] = carry;
    nonbinary = __any_sync(0xffffffffu, nonbinary);
    __syncwarp();
    double* dst = out + (size_t)row * nx_out;
    for (int xo = lane; xo < nx_out; xo += 32) {
      double acc = 0.0;
      if (xo >= si.lo && xo < si.hi) {
        const int e0 = S * xo + si.c0, e1 = e0 + NP;   // interior: 0 <= e0, e1 <= nx_in
        if (nonbinary) {
#pragma unroll
          for (int t = 0; t < NP; ++t) acc = __dadd_rn(acc, __dmul_rn(si.w[t], (double)bytes[e0 + t]));
        } else {
          const unsigned s0 = prefix[e0 >> 5] + __popc(words[e0 >> 5] & ((1u << (e0 & 31)) - 1u));
          const unsigned s1 = prefix[e1 >> 5] + ((e1 & 31) ? __popc(words[e1 >> 5] & ((1u << (e1 & 31)) - 1u)) : 0u);
          const unsigned cnt = s1 - s0;
          if (cnt == (unsigned)NP) {
            acc = si.wsum;
          } else if (cnt != 0) {
#pragma unroll
            for (int t = 0; t < NP; ++t)
              if (bytes[e0 + t]) acc = __dadd_rn(acc, si.w[t]);
          }
        }
      } else if (edge_tab) {
        const int k = xo < si.lo ? xo : si.lo + (xo - si.hi);
        for (int t = 0; t < NP; ++t)
          acc = __dadd_rn(acc, __dmul_rn(edge_w[k * NP + t], (double)bytes[edge_i[k * NP + t]]));
      } else {
        for (int t = 0; t < NP; ++t)
          acc = __dadd_rn(acc, __dmul_rn(__ldg(w + (size_t)t * nx_out + xo),
                                         (double)__ldg(src + __ldg(idx + (size_t)t * nx_out + xo))));
      }
      dst[xo] = acc;
    }
    __syncwarp();
  }
}

// out[z][yo][x] = sum_t w[yo][t] * in[z][idx[yo][t]][x]
template <typename Tin, typename A, typename Tout>
__global__ void k_resample_y(const __grid_constant__ SITaps si, const Tin* __restrict__ in, Tout* __restrict__ out,
                             int nz, int ny_in, int ny_out, int nx, const double* __restrict__ w,
                             const int32_t* __restrict__ idx, int P, int stride, int comp) {
  const size_t rs = (size_t)nx * stride;   // input row stride
  WR_FOR_ROWS(nz * ny_out, row) {
    const int z = row / ny_out, yo = row - z * ny_out;
    const Tin* plane = in + (size_t)z * ny_in * rs + comp;
    Tout* dst = out + (size_t)row * nx;
    if (yo >= si.lo && yo < si.hi) {
      const Tin* r0 = plane + (size_t)(si.s * yo + si.c0) * rs;
      WR_FOR_COLS(nx, x) {
        const Tin* q = r0 + (size_t)x * stride;
        A acc = 0;
#pragma unroll 4
        for (int t = 0; t < si.P; ++t) acc = Acc<A>::madd(acc, Acc<A>::si_weight(si, t), (A)__ldg(q + (size_t)t * rs));
        dst[x] = (Tout)acc;
      }
    } else {
      const double* wr = w + (size_t)yo * P;
      const int32_t* ir = idx + (size_t)yo * P;
      WR_FOR_COLS(nx, x) {
        const Tin* q = plane + (size_t)x * stride;
        A acc = 0;
        for (int t = 0; t < P; ++t) acc = Acc<A>::madd(acc, __ldg(wr + t), (A)__ldg(q + (size_t)__ldg(ir + t) * rs));
        dst[x] = (Tout)acc;
      }
    }
  }
}

// The y pass for an integer down-scale factor S (P = 4S + 2 taps fixed at
// compile time, weights as constant operands); rows outside the
// shift-invariant interior read the table.
template <int S, typename Tin, typename A, typename Tout>
__global__ void k_resample_y_si(const __grid_constant__ SITaps si, const Tin* __restrict__ in,
                                Tout* __restrict__ out, int nz, int ny_in, int ny_out, int nx,
                                const double* __restrict__ w, const int32_t* __restrict__ idx) {
  constexpr int NP = 4 * S + 2;
  WR_FOR_ROWS(nz * ny_out, row) {
    const int z = row / ny_out, yo = row - z * ny_out;
    const Tin* plane = in + (size_t)z * ny_in * nx;
    Tout* dst = out + (size_t)row * nx;
    if (yo >= si.lo && yo < si.hi) {
      const Tin* r0 = plane + (size_t)(S * yo + si.c0) * nx;
      WR_FOR_COLS(nx, x) {
        A v[NP];
#pragma unroll
        for (int t = 0; t < NP; ++t) v[t] = (A)__ldg(r0 + (size_t)t * nx + x);
        A acc = 0;
#pragma unroll
        for (int t = 0; t < NP; ++t) acc = Acc<A>::madd(acc, Acc<A>::si_weight(si, t), v[t]);
        dst[x] = (Tout)acc;
      }
    } else {
      const double* wr = w + (size_t)yo * NP;
      const int32_t* ir = idx + (size_t)yo * NP;
      WR_FOR_COLS(nx, x) {
        A acc = 0;
        for (int t = 0; t < NP; ++t) acc = Acc<A>::madd(acc, __ldg(wr + t), (A)__ldg(plane + (size_t)__ldg(ir + t) * nx + x));
        dst[x] = (Tout)acc;
      }
    }
  }
}

// The y pass with V adjacent columns per lane: each tap row is one vector
// load of V inputs (V times fewer loads in flight for the same bytes), the V
// outputs summed in tap order as in k_resample_y_si.  Rows whose length is a
// multiple of V with the row starts aligned to V elements; edge output rows
// read the table.
template <int S, int V, typename Tin, typename A, typename Tout>
__global__ void k_resample_y_si_v(const __grid_constant__ SITaps si, const Tin* __restrict__ in,
                                  Tout* __restrict__ out, int nz, int ny_in, int ny_out, int nx,
                                  const double* __restrict__ w, const int32_t* __restrict__ idx) {
  constexpr int NP = 4 * S + 2;
  const int ng = nx / V;
  WR_FOR_ROWS(nz * ny_out, row) {
    const int z = row / ny_out, yo = row - z * ny_out;
    const Tin* plane = in + (size_t)z * ny_in * nx;
    Tout* dst = out + (size_t)row * nx;
    if (yo >= si.lo && yo < si.hi) {
      const Tin* r0 = plane + (size_t)(S * yo + si.c0) * nx;
      WR_FOR_COLS(ng, xg) {
        A acc[V];
#pragma unroll
        for (int c = 0; c < V; ++c) acc[c] = 0;
#pragma unroll
        for (int t = 0; t < NP; ++t) {
          Tin v[V];
          load_group<Tin, V>(r0 + (size_t)t * nx + V * xg, v);
#pragma unroll
          for (int c = 0; c < V; ++c) acc[c] = Acc<A>::madd(acc[c], Acc<A>::si_weight(si, t), (A)v[c]);
        }
#pragma unroll
        for (int c = 0; c < V; ++c) dst[V * xg + c] = (Tout)acc[c];
      }
    } else {
      const double* wr = w + (size_t)yo * NP;
      const int32_t* ir = idx + (size_t)yo * NP;
      WR_FOR_COLS(nx, x) {
        A acc = 0;
        for (int t = 0; t < NP; ++t) acc = Acc<A>::madd(acc, __ldg(wr + t), (A)__ldg(plane + (size_t)__ldg(ir + t) * nx + x));
        dst[x] = (Tout)acc;
      }
    }
  }
}

// uint8 mask -> float64 0/1 (first pass input for the float64 mask resize)
__global__ void k_mask_to_d(const uint8_t* __restrict__ m, double* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = m[i] ? 1.0 : 0.0;
}

// ---------------------------------------------------------------------------
// level packing
// ---------------------------------------------------------------------------

template <typename T, typename O>
__global__ void k_to_float(const T* __restrict__ in, O* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (O)load_f<T>(in, i);
}

// input volume -> stored reference level (level 0: the resize is a copy)
template <typename T, int PREC>
__global__ void k_to_level(const T* __restrict__ in, typename Store<PREC>::V1* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = Store<PREC>::pack1(load_f<T>(in, i));
}

// float level -> stored reference level
template <int PREC>
__global__ void k_store_level(const float* __restrict__ in, typename Store<PREC>::V1* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = Store<PREC>::pack1(in[i]);
}

// movg[p] = (m, Gx, Gy, Gz) with G = half the clamped central difference.
// Each warp takes 32 columns of a row; the x neighbours come from the
// adjacent lanes.
template <typename T, int PREC>
__global__ void k_pack_movg(const T* __restrict__ m, typename Store<PREC>::V4* __restrict__ movg, int nz, int ny, int nx) {
  const size_t sy = nx, sz = (size_t)nx * ny;
  const int lane = threadIdx.x;
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    const size_t base = (size_t)row * nx;
    const size_t dyp = (size_t)(min(y + 1, ny - 1) - y) * sy, dym = (size_t)(y - max(y - 1, 0)) * sy;
    const size_t dzp = (size_t)(min(z + 1, nz - 1) - z) * sz, dzm = (size_t)(z - max(z - 1, 0)) * sz;
    for (int x0 = 0; x0 < nx; x0 += 32) {
      const int x = x0 + lane, xc = min(x, nx - 1);
      const size_t i = base + xc;
      const float c = load_f<T>(m, i);
      float xm = __shfl_up_sync(0xffffffffu, c, 1), xp = __shfl_down_sync(0xffffffffu, c, 1);
      if (lane == 0) xm = load_f<T>(m, base + max(xc - 1, 0));
      if (lane == 31 || x >= nx - 1) xp = load_f<T>(m, base + min(xc + 1, nx - 1));
      if (x < nx) {
        const float yp = load_f<T>(m, i + dyp), ym = load_f<T>(m, i - dym);
        const float zp = load_f<T>(m, i + dzp), zm = load_f<T>(m, i - dzm);
        movg[i] = Store<PREC>::pack4(make_float4(c, 0.5f * (xp - xm), 0.5f * (yp - ym), 0.5f * (zp - zm)));
      }
    }
  }
}

// mask bits of a level: bit0 = resized mask_ref > 0; bits 1-2 = class of the
// trilinear cell whose lower corner is this voxel in the resized mask_mov:
// 0 = all 8 corners <= 0, 1 = all > 0, 2 = mixed (needs the exact sum).
// Four consecutive elements of a row (16-byte loads for float, 8 for
// uint16, 4 for uint8; the caller checks the alignment).
template <typename T> __device__ __forceinline__ float4 load_x4(const T* p);
template <> __device__ __forceinline__ float4 load_x4<float>(const float* p) {
  return __ldg(reinterpret_cast<const float4*>(p));
}
template <> __device__ __forceinline__ float4 load_x4<uint16_t>(const uint16_t* p) {
  const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
  return make_float4((float)(v.x & 0xffffu), (float)(v.x >> 16), (float)(v.y & 0xffffu), (float)(v.y >> 16));
}
template <> __device__ __forceinline__ float4 load_x4<uint8_t>(const uint8_t* p) {
  const unsigned v = __ldg(reinterpret_cast<const unsigned*>(p));
  return make_float4((float)(v & 0xffu), (float)((v >> 8) & 0xffu), (float)((v >> 16) & 0xffu), (float)(v >> 24));
}

// k_pack_movg with four voxels per lane (nx a multiple of 4, rows aligned
// for load_x4): one 4-wide load per neighbouring row, the x neighbours from
// the lane's own elements and the adjacent lanes.
template <typename T, int PREC>
__global__ void k_pack_movg_x4(const T* __restrict__ m, typename Store<PREC>::V4* __restrict__ movg, int nz, int ny,
                               int nx) {
  const size_t sy = nx, sz = (size_t)nx * ny;
  const int lane = threadIdx.x;
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    const size_t base = (size_t)row * nx;
    const size_t dyp = (size_t)(min(y + 1, ny - 1) - y) * sy, dym = (size_t)(y - max(y - 1, 0)) * sy;
    const size_t dzp = (size_t)(min(z + 1, nz - 1) - z) * sz, dzm = (size_t)(z - max(z - 1, 0)) * sz;
    float carry = 0.f;   // last element of the previous chunk
    for (int x0 = 0; x0 < nx; x0 += 128) {
      const int x = x0 + 4 * lane, xc = min(x, nx - 4);
      const size_t i = base + xc;
      const float4 c = load_x4<T>(m + i);
      const float4 yp = load_x4<T>(m + i + dyp), ym = load_x4<T>(m + i - dym);
      const float4 zp = load_x4<T>(m + i + dzp), zm = load_x4<T>(m + i - dzm);
      const float ahead = load_f<T>(m, base + min(x0 + 128, nx - 1));   // same address in every lane
      float left = __shfl_up_sync(0xffffffffu, c.w, 1);
      float right = __shfl_down_sync(0xffffffffu, c.x, 1);
      if (lane == 0) left = x0 == 0 ? c.x : carry;
      if (lane == 31) right = ahead;
      if (x + 4 >= nx) right = c.w;
      carry = __shfl_sync(0xffffffffu, c.w, 31);
      if (x < nx) {
        typename Store<PREC>::V4* o = movg + base + x;
        o[0] = Store<PREC>::pack4(make_float4(c.x, 0.5f * (c.y - left), 0.5f * (yp.x - ym.x), 0.5f * (zp.x - zm.x)));
        o[1] = Store<PREC>::pack4(make_float4(c.y, 0.5f * (c.z - c.x), 0.5f * (yp.y - ym.y), 0.5f * (zp.y - zm.y)));
        o[2] = Store<PREC>::pack4(make_float4(c.z, 0.5f * (c.w - c.y), 0.5f * (yp.z - ym.z), 0.5f * (zp.z - zm.z)));
        o[3] = Store<PREC>::pack4(make_float4(c.w, 0.5f * (right - c.z), 0.5f * (yp.w - ym.w), 0.5f * (zp.w - zm.w)));
      }
    }
  }
}

// k_mask_bits for full-resolution uint8 masks with four voxels per lane (nx a
// multiple of 4, rows 4-byte aligned); same bits and float moving mask.
__global__ void k_mask_bits_u8x4(const uint8_t* __restrict__ mref_u8, const uint8_t* __restrict__ mmov,
                                 float* __restrict__ mmov_f, uint8_t* __restrict__ bits, int nz, int ny, int nx,
                                 int keep_ref_bit) {
  const int lane = threadIdx.x;
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    const size_t base = (size_t)row * nx;
    const size_t dy = (size_t)(min(y + 1, ny - 1) - y) * nx, dz = (size_t)(min(z + 1, nz - 1) - z) * nx * ny;
    for (int x0 = 0; x0 < nx; x0 += 128) {
      const int x = x0 + 4 * lane, xc = min(x, nx - 4);
      const size_t i = base + xc;
      unsigned b = 0;
      if (keep_ref_bit) b = __ldg(reinterpret_cast<const unsigned*>(bits + i)) & 0x01010101u;
      else if (mref_u8) {
        const unsigned r = __ldg(reinterpret_cast<const unsigned*>(mref_u8 + i));
        b = __vcmpne4(r, 0u) & 0x01010101u;   // bit 0 of each byte: nonzero
      }
      if (mmov) {
        // per row of the cell (y, z), (y+1, z), (y, z+1), (y+1, z+1): 4 nonzero flags in bits 0..3
        unsigned fl[4];
        const size_t offs[4] = {0, dy, dz, dz + dy};
        const size_t ahead = base + min(x0 + 128, nx - 1);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const unsigned v = __ldg(reinterpret_cast<const unsigned*>(mmov + i + offs[r]));
          // nonzero flags of bytes 0..3 gathered into bits 0..3
          const unsigned f = ((__vcmpne4(v, 0u) & 0x01010101u) * 0x01020408u) >> 24;
          unsigned nxt = __shfl_down_sync(0xffffffffu, f, 1) & 1u;          // next lane's first element
          if (lane == 31) nxt = __ldg(mmov + ahead + offs[r]) != 0 ? 1u : 0u;
          if (x + 4 >= nx) nxt = (f >> 3) & 1u;                             // edge clamp
          fl[r] = f | (nxt << 4);
        }
        float mf[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const unsigned pair = 3u << j;   // columns j, j+1
          const unsigned any = (fl[0] | fl[1] | fl[2] | fl[3]) & pair;
          const unsigned all = (fl[0] & fl[1] & fl[2] & fl[3]) & pair;
          const unsigned code = any == 0 ? 0u : (all == pair ? 1u : 2u);
          b |= code << (8 * j + 1);
          mf[j] = (fl[0] >> j) & 1u ? 1.f : 0.f;
        }
        if (mmov_f && x < nx) *reinterpret_cast<float4*>(mmov_f + base + x) = make_float4(mf[0], mf[1], mf[2], mf[3]);
      }
      if (x < nx) *reinterpret_cast<unsigned*>(bits + base + x) = b;
    }
  }
}

// k_mask_bits for levels >= 1 (float64 reference mask, float moving mask)
// with four voxels per lane (nx a multiple of 4, rows 16-byte aligned): the
// same bits, with 16-byte loads and the x + 1 corners from the next lane.
__global__ void k_mask_bits_f4(const double* __restrict__ mref_d, const float* __restrict__ mmov,
                               uint8_t* __restrict__ bits, int nz, int ny, int nx, int keep_ref_bit) {
  const int lane = threadIdx.x;
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    const size_t base = (size_t)row * nx;
    const size_t dy = (size_t)(min(y + 1, ny - 1) - y) * nx, dz = (size_t)(min(z + 1, nz - 1) - z) * nx * ny;
    for (int x0 = 0; x0 < nx; x0 += 128) {
      const int x = x0 + 4 * lane, xc = min(x, nx - 4);
      const size_t i = base + xc;
      unsigned b = 0;
      if (keep_ref_bit) {
        b = __ldg(reinterpret_cast<const unsigned*>(bits + i)) & 0x01010101u;
      } else if (mref_d) {
        const double2 r0 = __ldg(reinterpret_cast<const double2*>(mref_d + i));
        const double2 r1 = __ldg(reinterpret_cast<const double2*>(mref_d + i) + 1);
        b = (r0.x > 0.0 ? 1u : 0u) | (r0.y > 0.0 ? 0x100u : 0u) | (r1.x > 0.0 ? 0x10000u : 0u) |
            (r1.y > 0.0 ? 0x1000000u : 0u);
      }
      if (mmov) {
        // per row of the cell (y, z), (y+1, z), (y, z+1), (y+1, z+1): 4 flags in bits 0..3
        unsigned fl[4];
        const size_t offs[4] = {0, dy, dz, dz + dy};
        const size_t ahead = base + min(x0 + 128, nx - 1);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const float4 v = __ldg(reinterpret_cast<const float4*>(mmov + i + offs[r]));
          const unsigned f = (v.x > 0.f ? 1u : 0u) | (v.y > 0.f ? 2u : 0u) | (v.z > 0.f ? 4u : 0u) | (v.w > 0.f ? 8u : 0u);
          unsigned nxt = __shfl_down_sync(0xffffffffu, f, 1) & 1u;          // next lane's first element
          if (lane == 31) nxt = __ldg(mmov + ahead + offs[r]) > 0.f ? 1u : 0u;
          if (x + 4 >= nx) nxt = (f >> 3) & 1u;                             // edge clamp
          fl[r] = f | (nxt << 4);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const unsigned pair = 3u << j;   // columns j, j+1
          const unsigned any = (fl[0] | fl[1] | fl[2] | fl[3]) & pair;
          const unsigned all = (fl[0] & fl[1] & fl[2] & fl[3]) & pair;
          const unsigned code = any == 0 ? 0u : (all == pair ? 1u : 2u);
          b |= code << (8 * j + 1);
        }
      }
      if (x < nx) *reinterpret_cast<unsigned*>(bits + base + x) = b;
    }
  }
}

template <typename TM> __device__ __forceinline__ bool mask_on(const TM* m, size_t i);
template <> __device__ __forceinline__ bool mask_on<float>(const float* m, size_t i) { return __ldg(m + i) > 0.f; }
template <> __device__ __forceinline__ bool mask_on<uint8_t>(const uint8_t* m, size_t i) { return __ldg(m + i) != 0; }

// Exclusion bits of a level: bit 0 = reference mask > 0 (from its float64
// resize, its uint8 values at full resolution, or kept), bits 1-2 = class
// of the moving mask's trilinear cell at each voxel (corners x..x+1,
// y..y+1, z..z+1, edge-clamped): 0 no corner > 0, 1 all, 2 mixed.  Each warp
// takes 32 columns of a row; the x+1 corners come from the next lane's
// ballot bit.  mmov_f (optional) receives the moving mask as float (the
// full-resolution level, where TM is uint8).
template <typename TM>
__global__ void k_mask_bits(const double* __restrict__ mref_d, const uint8_t* __restrict__ mref_u8,
                            const TM* __restrict__ mmov, float* __restrict__ mmov_f, uint8_t* __restrict__ bits,
                            int nz, int ny, int nx, int keep_ref_bit) {
  const int lane = threadIdx.x;
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    const size_t base = (size_t)row * nx;
    const size_t dy = (size_t)(min(y + 1, ny - 1) - y) * nx, dz = (size_t)(min(z + 1, nz - 1) - z) * nx * ny;
    for (int x0 = 0; x0 < nx; x0 += 32) {
      const int x = x0 + lane, xc = min(x, nx - 1);
      const size_t i = base + xc;
      uint8_t b = 0;
      if (x < nx) {
        b = keep_ref_bit ? (bits[i] & 1) : 0;
        if (mref_d) b |= (mref_d[i] > 0.0) ? 1 : 0;
        else if (mref_u8) b |= mref_u8[i] ? 1 : 0;
      }
      if (mmov) {
        const bool f0 = mask_on<TM>(mmov, i), f1 = mask_on<TM>(mmov, i + dy);
        const bool f2 = mask_on<TM>(mmov, i + dz), f3 = mask_on<TM>(mmov, i + dz + dy);
        const unsigned b0 = __ballot_sync(0xffffffffu, f0), b1 = __ballot_sync(0xffffffffu, f1);
        const unsigned b2 = __ballot_sync(0xffffffffu, f2), b3 = __ballot_sync(0xffffffffu, f3);
        bool n0, n1, n2, n3;   // corners at column min(x + 1, nx - 1)
        if (x >= nx - 1) {
          n0 = f0; n1 = f1; n2 = f2; n3 = f3;
        } else if (lane == 31) {
          const size_t j = base + x + 1;
          n0 = mask_on<TM>(mmov, j); n1 = mask_on<TM>(mmov, j + dy);
          n2 = mask_on<TM>(mmov, j + dz); n3 = mask_on<TM>(mmov, j + dz + dy);
        } else {
          n0 = (b0 >> (lane + 1)) & 1u; n1 = (b1 >> (lane + 1)) & 1u;
          n2 = (b2 >> (lane + 1)) & 1u; n3 = (b3 >> (lane + 1)) & 1u;
        }
        const bool any = f0 | f1 | f2 | f3 | n0 | n1 | n2 | n3;
        const bool all = f0 & f1 & f2 & f3 & n0 & n1 & n2 & n3;
        b |= (uint8_t)((any ? (all ? 1 : 2) : 0) << 1);
        if (mmov_f && x < nx) mmov_f[i] = f0 ? 1.f : 0.f;
      }
      if (x < nx) bits[i] = b;
    }
  }
}

__global__ void k_d_to_f(const double* __restrict__ in, float* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

// ---------------------------------------------------------------------------
// motion field evaluation
// ---------------------------------------------------------------------------

struct CPView {
  const float4* cp;
  int ncx, ncy, r, w;
};

// Dense motion of a voxel from the CP grid: trilinear map_coordinates on the
// CP grid at ((x-r)/(2r+1), (y-r)/(2r+1), z), coordinates clamped to
// [0, ncp] then taps edge-clamped (utils/calFlow3d_Wei_v1.py:265-292,626-640).
__device__ __forceinline__ float3 cp_field(const CPView& g, int x, int y, int z) {
  float gx = __fdiv_rn((float)(x - g.r), (float)g.w);
  float gy = __fdiv_rn((float)(y - g.r), (float)g.w);
  gx = fminf(fmaxf(gx, 0.f), (float)g.ncx);
  gy = fminf(fmaxf(gy, 0.f), (float)g.ncy);
  float fx = floorf(gx), fy = floorf(gy);
  float tx = gx - fx, ty = gy - fy;
  int ix0 = min((int)fx, g.ncx - 1), ix1 = min((int)fx + 1, g.ncx - 1);
  int iy0 = min((int)fy, g.ncy - 1), iy1 = min((int)fy + 1, g.ncy - 1);
  const float4* b = g.cp + (size_t)z * g.ncy * g.ncx;
  float4 a00 = b[iy0 * g.ncx + ix0], a01 = b[iy0 * g.ncx + ix1];
  float4 a10 = b[iy1 * g.ncx + ix0], a11 = b[iy1 * g.ncx + ix1];
  float w00 = (1.f - tx) * (1.f - ty), w01 = tx * (1.f - ty), w10 = (1.f - tx) * ty, w11 = tx * ty;
  float3 r;
  r.x = w00 * a00.x + w01 * a01.x + w10 * a10.x + w11 * a11.x;
  r.y = w00 * a00.y + w01 * a01.y + w10 * a10.y + w11 * a11.y;
  r.z = w00 * a00.z + w01 * a01.z + w10 * a10.z + w11 * a11.z;
  return r;
}

// Up-sampled field of the previous (coarser) level: bilinear imresize of its
// dense field, x and y components doubled (utils/calFlow3d_Wei_v1.py:381-410).
struct UpView {
  CPView src;                 // coarser level's CP grid
  const float4* src_dense;    // or its dense field (used when non-null)
  int src_nx, src_ny;
  const float* wx; const int32_t* ix;
  const float* wy; const int32_t* iy;
  int x_first;
};

__device__ __forceinline__ float3 coarse_value(const UpView& u, int x, int y, int z) {
  if (u.src_dense) {
    float4 v = u.src_dense[((size_t)z * u.src_ny + y) * u.src_nx + x];
    return make_float3(v.x, v.y, v.z);
  }
  return cp_field(u.src, x, y, z);
}

__device__ __forceinline__ float3 up_field(const UpView& u, int x, int y, int z) {
  float wx0 = u.wx[2 * x], wx1 = u.wx[2 * x + 1];
  int ix0 = u.ix[2 * x], ix1 = u.ix[2 * x + 1];
  float wy0 = u.wy[2 * y], wy1 = u.wy[2 * y + 1];
  int iy0 = u.iy[2 * y], iy1 = u.iy[2 * y + 1];
  float3 f00 = coarse_value(u, ix0, iy0, z), f01 = coarse_value(u, ix1, iy0, z);
  float3 f10 = coarse_value(u, ix0, iy1, z), f11 = coarse_value(u, ix1, iy1, z);
  float3 r;
  if (u.x_first) {
    float3 r0 = make_float3(wx0 * f00.x + wx1 * f01.x, wx0 * f00.y + wx1 * f01.y, wx0 * f00.z + wx1 * f01.z);
    float3 r1 = make_float3(wx0 * f10.x + wx1 * f11.x, wx0 * f10.y + wx1 * f11.y, wx0 * f10.z + wx1 * f11.z);
    r = make_float3(wy0 * r0.x + wy1 * r1.x, wy0 * r0.y + wy1 * r1.y, wy0 * r0.z + wy1 * r1.z);
  } else {
    float3 c0 = make_float3(wy0 * f00.x + wy1 * f10.x, wy0 * f00.y + wy1 * f10.y, wy0 * f00.z + wy1 * f10.z);
    float3 c1 = make_float3(wy0 * f01.x + wy1 * f11.x, wy0 * f01.y + wy1 * f11.y, wy0 * f01.z + wy1 * f11.z);
    r = make_float3(wx0 * c0.x + wx1 * c1.x, wx0 * c0.y + wx1 * c1.y, wx0 * c0.z + wx1 * c1.z);
  }
  r.x *= 2.f;
  r.y *= 2.f;
  return r;
}

struct FieldSrc {
  int mode;            // FieldMode
  CPView cpv;          // FIELD_CP
  UpView up;           // FIELD_UP
  const float4* dense; // FIELD_DENSE
  int nx, ny;
};

template <int MODE>
__device__ __forceinline__ float3 eval_field(const FieldSrc& f, int x, int y, int z) {
  if (MODE == FIELD_CP) return cp_field(f.cpv, x, y, z);
  if (MODE == FIELD_UP) return up_field(f.up, x, y, z);
  if (MODE == FIELD_DENSE) {
    float4 v = f.dense[((size_t)z * f.ny + y) * f.nx + x];
    return make_float3(v.x, v.y, v.z);
  }
  return make_float3(0.f, 0.f, 0.f);
}

// ---------------------------------------------------------------------------
// trilinear sampling
// ---------------------------------------------------------------------------

struct VolView {
  const void* g;     // (m, Gx, Gy, Gz) in the storage of the call's precision
  int nx, ny, nz;
};

// float64 trilinear of a float32 volume, cast to float32 (scipy's arithmetic
// for the warped exclusion mask).
__device__ __forceinline__ float sample_f64(const float* v, int nx, int ny, int nz, float cx, float cy, float cz) {
  int x0, y0, z0;
  float tx_f, ty_f, tz_f;
  split_coord(cx, x0, tx_f);
  split_coord(cy, y0, ty_f);
  split_coord(cz, z0, tz_f);
  double tx = tx_f, ty = ty_f, tz = tz_f;
  int xs[2] = {clampi(x0, 0, nx - 1), clampi(x0 + 1, 0, nx - 1)};
  int ys[2] = {clampi(y0, 0, ny - 1), clampi(y0 + 1, 0, ny - 1)};
  int zs[2] = {clampi(z0, 0, nz - 1), clampi(z0 + 1, 0, nz - 1)};
  double acc = 0.0;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        double wgt = (a ? tx : 1.0 - tx) * (b ? ty : 1.0 - ty) * (c ? tz : 1.0 - tz);
        acc += wgt * (double)v[((size_t)zs[c] * ny + ys[b]) * nx + xs[a]];
      }
  return (float)acc;
}

// ---------------------------------------------------------------------------
// block reductions
// ---------------------------------------------------------------------------

template <int N>
__device__ __forceinline__ void block_sum(float (&v)[N], float* red /* [32*N] */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < N; ++k) red[warp * N + k] = v[k];
  __syncthreads();
  if (threadIdx.x < N) {
    float s = 0.f;
    for (int wi = 0; wi < nw; ++wi) s += red[wi * N + threadIdx.x];
    red[32 * N + threadIdx.x] = s;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = red[32 * N + k];
}

__device__ __forceinline__ float block_max(float v, float* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = 0.f;
    for (int wi = 0; wi < nw; ++wi) m = fmaxf(m, red[wi]);
    red[32] = m;
  }
  __syncthreads();
  return red[32];
}

// ---------------------------------------------------------------------------
// fused LK iteration: warp + masked smoothed It + gradients + window sums
// (utils/calFlow3d_Wei_v1.py:442-588)
// ---------------------------------------------------------------------------

__device__ __forceinline__ float3 lerp3(const float3& a, const float3& b, float t) {
  return make_float3(fmaf(t, b.x - a.x, a.x), fmaf(t, b.y - a.y, a.y), fmaf(t, b.z - a.z, a.z));
}
__device__ __forceinline__ float4 lerp4(const float4& a, const float4& b, float t) {
  return make_float4(fmaf(t, b.x - a.x, a.x), fmaf(t, b.y - a.y, a.y), fmaf(t, b.z - a.z, a.z),
                     fmaf(t, b.w - a.w, a.w));
}

// floor(n / d) by a multiply-high: m = ceil(2^32 / d) gives the exact
// quotient for every n >= 0 with n * d <= 2^32 (n = qd + r: the product
// n m / 2^32 exceeds n / d by n e / (d 2^32), e = m d - 2^32 < d, which keeps
// it below q + 1).  m = 0 marks a divisor without a multiplier (d = 1 or the
// bound not met); host_div_magic computes m.
__device__ __forceinline__ int div_magic(int n, int d, uint32_t m) {
  return m ? (int)__umulhi((uint32_t)n, m) : (d == 1 ? n : n / d);
}

// floor(n / d) for 0 <= n < 4096 and 1 <= d < 4096: (n + 0.5) / d is at least
// 0.5 / d away from the integers on either side, far more than the error of
// the approximate float quotient, so truncating it is exact.
__device__ __forceinline__ int div_small(int n, int d) {
  return (int)__fdividef((float)n + 0.5f, (float)d);
}

struct IterArgs {
  LKState* st;
  const void* __restrict__ ref;        // reference level in the call's storage
  VolView mov;
  const uint8_t* __restrict__ mbits;   // null: no masks
  const float* __restrict__ mmov;      // null: no moving mask
  float* __restrict__ sums;            // ncp * 12: 9 window sums + 3 neighbour differences
  double* __restrict__ errpart;        // per CTA
  double* __restrict__ penpart;        // per CTA
  CPView cpv;                          // this level's CPs (motion_current at CPs)
  FieldSrc field;                      // motion used for this iteration
  FieldSrc field0;                     // level's initial field (first-diff launches)
  int r, w, ntx, nty;
  float zratio;
  uint32_t nz_magic, ntx_magic;        // div_magic multipliers of nz and ntx for the tile indexes
  // level constants of the sampling loop, read as kernel parameters rather
  // than recomputed from nx, ny, nz in the loop
  int nxm1, nym1, nxm2, nym2, bzmax;
  uint32_t plane, oz1;
  float fnx, fny, fnz, fnxm1, fnym1, fnzm1, fzmax;
};

// warped moving exclusion mask > 0, evaluated exactly (float64 sum, float32 result)
__device__ __noinline__ bool warped_mask_exact(const float* mmov, int nx, int ny, int nz, float cx, float cy, float cz) {
  return sample_f64(mmov, nx, ny, nz, cx, cy, cz) > 0.f;
}

// CP-grid interpolation factors along one axis: the (g - r)/(2r+1) coordinate
// clamped to [0, ncp] (utils/calFlow3d_Wei_v1.py:265-292), lower / upper CP
// index (absolute, edge-clamped) and fraction.
__device__ __forceinline__ int2 cp_factor(int g, int r, int w, int ncp, float& t) {
  float c = __fdiv_rn((float)(g - r), (float)w);
  c = fminf(fmaxf(c, 0.f), (float)ncp);
  const float f = floorf(c);
  t = c - f;
  return make_int2(min((int)f, ncp - 1), min((int)f + 1, ncp - 1));
}

constexpr int kAccThreads = 256;
constexpr int kTileCP = 4;   // CP rows / columns held per tile

// Motion of a (w+2) x (w+2) tile from shared memory: motion(hx, hy) =
// sum_j wy[hy].j * ax[hx][j], where ax holds the CP field interpolated along x
// for kTileCP CP rows and wy the y weights of those rows.  For the up-sampled
// field of a level's first iteration (utils/calFlow3d_Wei_v1.py:381-410) the
// same separable form holds over the coarser level's CPs: the bilinear
// up-sampling table composed with that level's CP interpolation, x and y
// components doubled.
//
// ax is stored CP row by CP row ([kTileCP][ld]) so that the lanes of a warp,
// which hold consecutive columns, read consecutive float4s (no shared-memory
// bank conflicts).  In CP mode a row of the tile touches at most two CP rows:
// wy[hy] then holds their weights and row indexes (w0, w1, j0, j1); in UP
// mode it holds the four row weights.
struct TileField {
  float4* ax;   // [kTileCP][ld]
  float4* wy;   // [hh]
  float4* cpt;  // [kTileCP][kTileCP]
  int ld;       // row length of ax (w + 2)
};

__host__ __device__ inline size_t tile_field_smem(int w) {
  return 16 * ((size_t)(w + 2) * kTileCP + (w + 2) + kTileCP * kTileCP) + 16;
}

// Fills the tile field for MODE (all threads of the CTA call it; ends with a barrier).
template <int MODE>
__device__ void build_tile_field(const TileField& tf, int* generic_flag, const FieldSrc& f, int r, int w, int x0,
                                 int y0, int hw, int hh, int z, int nx, int ny) {
  if (threadIdx.x == 0) *generic_flag = 0;
  if (MODE == FIELD_CP) {
    const CPView& g = f.cpv;
    float t;
    if (threadIdx.x < 32) {
      // one warp finds the CP tile origin (the lowest CP index used by the
      // tile's first column / row) and loads the CP tile
      const int cx0 = cp_factor(clampi(x0 - 1, 0, nx - 1), r, w, g.ncx, t).x;
      const int cy0 = cp_factor(clampi(y0 - 1, 0, ny - 1), r, w, g.ncy, t).x;
      if (threadIdx.x == 0) { generic_flag[2] = cx0; generic_flag[3] = cy0; }
      if (threadIdx.x < kTileCP * kTileCP) {
        const int jr = threadIdx.x / kTileCP, jc = threadIdx.x % kTileCP;
        tf.cpt[threadIdx.x] = g.cp[((size_t)z * g.ncy + min(cy0 + jr, g.ncy - 1)) * g.ncx + min(cx0 + jc, g.ncx - 1)];
      }
    }
    __syncthreads();
    const int cx0 = generic_flag[2], cy0 = generic_flag[3];
    if (threadIdx.x < hw) {
      const int gx = clampi(x0 - 1 + (int)threadIdx.x, 0, nx - 1);
      const int2 c = cp_factor(gx, r, w, g.ncx, t);
      const int i0 = c.x - cx0, i1 = c.y - cx0;
      for (int j = 0; j < kTileCP; ++j) {
        const float4 p = tf.cpt[j * kTileCP + min(i0, kTileCP - 1)], q = tf.cpt[j * kTileCP + min(i1, kTileCP - 1)];
        tf.ax[j * tf.ld + threadIdx.x] =
            make_float4(fmaf(t, q.x - p.x, p.x), fmaf(t, q.y - p.y, p.y), fmaf(t, q.z - p.z, p.z), 0.f);
      }
      if (i1 >= kTileCP) atomicOr(generic_flag, 1);
    }
    if (threadIdx.x >= 128 && threadIdx.x < 128 + hh) {
      const int hy = threadIdx.x - 128;
      const int gy = clampi(y0 - 1 + hy, 0, ny - 1);
      const int2 c = cp_factor(gy, r, w, g.ncy, t);
      const int j0 = min(c.x - cy0, kTileCP - 1), j1 = min(c.y - cy0, kTileCP - 1);
      if (c.y - cy0 >= kTileCP) atomicOr(generic_flag, 1);
      float w0 = 1.f - t, w1 = t;
      if (j0 == j1) { w0 = w0 + w1; w1 = 0.f; }   // both weights on one row (edge clamp)
      tf.wy[hy] = make_float4(w0, w1, __int_as_float(j0), __int_as_float(j1));
    }
  } else if (MODE == FIELD_UP) {
    const UpView& u = f.up;
    const CPView& g = u.src;
    float t;
    if (threadIdx.x < 32) {
      // one warp finds the coarse CP origin (lowest CP index reached from the
      // first column / row) and loads the CP tile
      const int gx0 = clampi(x0 - 1, 0, nx - 1), gy0 = clampi(y0 - 1, 0, ny - 1);
      int cx0 = cp_factor(u.ix[2 * gx0], r, w, g.ncx, t).x, cy0 = cp_factor(u.iy[2 * gy0], r, w, g.ncy, t).x;
      if (u.wx[2 * gx0 + 1] != 0.f) cx0 = min(cx0, cp_factor(u.ix[2 * gx0 + 1], r, w, g.ncx, t).x);
      if (u.wy[2 * gy0 + 1] != 0.f) cy0 = min(cy0, cp_factor(u.iy[2 * gy0 + 1], r, w, g.ncy, t).x);
      if (threadIdx.x == 0) { generic_flag[2] = cx0; generic_flag[3] = cy0; }
      if (threadIdx.x < kTileCP * kTileCP) {
        const int jr = threadIdx.x / kTileCP, jc = threadIdx.x % kTileCP;
        tf.cpt[threadIdx.x] = g.cp[((size_t)z * g.ncy + min(cy0 + jr, g.ncy - 1)) * g.ncx + min(cx0 + jc, g.ncx - 1)];
      }
    }
    __syncthreads();
    const int cx0 = generic_flag[2], cy0 = generic_flag[3];
    if (threadIdx.x < hw) {
      const int gx = clampi(x0 - 1 + (int)threadIdx.x, 0, nx - 1);
      float wv[kTileCP] = {0.f, 0.f, 0.f, 0.f};
      bool over = false;
      for (int k = 0; k < 2; ++k) {
        const float uw = u.wx[2 * gx + k];
        if (uw == 0.f) continue;
        const int2 c = cp_factor(u.ix[2 * gx + k], r, w, g.ncx, t);
        const int i0 = c.x - cx0, i1 = c.y - cx0;
        over |= i1 >= kTileCP || i0 < 0;
        wv[clampi(i0, 0, kTileCP - 1)] += uw * (1.f - t);
        wv[clampi(i1, 0, kTileCP - 1)] += uw * t;
      }
      if (over) atomicOr(generic_flag, 1);
      for (int j = 0; j < kTileCP; ++j) {
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int i = 0; i < kTileCP; ++i) {
          const float4 c = tf.cpt[j * kTileCP + i];
          a.x = fmaf(wv[i], c.x, a.x);
          a.y = fmaf(wv[i], c.y, a.y);
          a.z = fmaf(wv[i], c.z, a.z);
        }
        a.x *= 2.f;
        a.y *= 2.f;
        tf.ax[j * tf.ld + threadIdx.x] = a;
      }
    }
    if (threadIdx.x >= 128 && threadIdx.x < 128 + hh) {
      const int hy = threadIdx.x - 128;
      const int gy = clampi(y0 - 1 + hy, 0, ny - 1);
      float wv[kTileCP] = {0.f, 0.f, 0.f, 0.f};
      bool over = false;
      for (int k = 0; k < 2; ++k) {
        const float uw = u.wy[2 * gy + k];
        if (uw == 0.f) continue;
        const int2 c = cp_factor(u.iy[2 * gy + k], r, w, g.ncy, t);
        const int j0 = c.x - cy0, j1 = c.y - cy0;
        over |= j1 >= kTileCP || j0 < 0;
        wv[clampi(j0, 0, kTileCP - 1)] += uw * (1.f - t);
        wv[clampi(j1, 0, kTileCP - 1)] += uw * t;
      }
      if (over) atomicOr(generic_flag, 1);
      tf.wy[hy] = make_float4(wv[0], wv[1], wv[2], wv[3]);
    }
  }
  __syncthreads();
}

template <int MODE>
__device__ __forceinline__ float3 tile_motion(const TileField& tf, bool generic, const FieldSrc& f, int hx, int hy,
                                              int gx, int gy, int z) {
  if (MODE == FIELD_CP && !generic) {
    const float4 wv = tf.wy[hy];
    const float4 p = tf.ax[__float_as_int(wv.z) * tf.ld + hx], q = tf.ax[__float_as_int(wv.w) * tf.ld + hx];
    return make_float3(fmaf(wv.y, q.x, __fmul_rn(wv.x, p.x)), fmaf(wv.y, q.y, __fmul_rn(wv.x, p.y)),
                       fmaf(wv.y, q.z, __fmul_rn(wv.x, p.z)));
  }
  if (MODE == FIELD_UP && !generic) {
    const float4 wv = tf.wy[hy];
    const float4 a0 = tf.ax[hx], a1 = tf.ax[tf.ld + hx], a2 = tf.ax[2 * tf.ld + hx], a3 = tf.ax[3 * tf.ld + hx];
    return make_float3(fmaf(wv.w, a3.x, fmaf(wv.z, a2.x, fmaf(wv.y, a1.x, __fmul_rn(wv.x, a0.x)))),
                       fmaf(wv.w, a3.y, fmaf(wv.z, a2.y, fmaf(wv.y, a1.y, __fmul_rn(wv.x, a0.y)))),
                       fmaf(wv.w, a3.z, fmaf(wv.z, a2.z, fmaf(wv.y, a1.z, __fmul_rn(wv.x, a0.z)))));
  }
  return eval_field<MODE>(f, gx, gy, z);
}

// Bytes of dynamic shared memory of k_lk_accumulate for patch width w
// (diff_up: a second tile field for the level's up-sampled initial field).
__host__ __device__ inline size_t accumulate_smem(int w, bool diff_up = false) {
  const size_t hw = (size_t)w + 2;
  return 16 * (size_t)w * w                  // gradients + exclusion of the tile voxels
         + 4 * ((hw * hw + 3) & ~size_t(3))  // It_raw of tile + halo
         + tile_field_smem(w)                // motion factors
         + 4 * 8 * 12 + 16                   // reduction scratch, flags
         + (diff_up ? tile_field_smem(w) + 16 : 0);
}

constexpr int kNoDiff = -1;

// Shared-memory carve-up of the iteration kernel for patch width w.
struct AccSmem {
  float4* gsm;     // gradients + exclusion of the tile voxels, w*w
  float* it_raw;   // It_raw of tile + halo, (w+2)^2 padded to 4
  TileField tf;    // motion factors of the iteration's field
  int* flags;
  float* red;      // reduction scratch, 8 warps * 12
  TileField tf0;   // the level's up-sampled initial field (first-diff launches)
  int* flags0;
  __device__ AccSmem(float4* base, int w) {
    gsm = base;
    it_raw = reinterpret_cast<float*>(gsm + w * w);
    tf.ax = reinterpret_cast<float4*>(it_raw + (((w + 2) * (w + 2) + 3) & ~3));
    tf.wy = tf.ax + (w + 2) * kTileCP;
    tf.cpt = tf.wy + (w + 2);
    tf.ld = w + 2;
    flags = reinterpret_cast<int*>(tf.cpt + kTileCP * kTileCP);
    red = reinterpret_cast<float*>(flags + 4);
    tf0.ax = reinterpret_cast<float4*>(red + 8 * 12);
    tf0.wy = tf0.ax + (w + 2) * kTileCP;
    tf0.cpt = tf0.wy + (w + 2);
    tf0.ld = w + 2;
    flags0 = reinterpret_cast<int*>(tf0.cpt + kTileCP * kTileCP);
  }
};

// Canonical index of the k-th tile visited: tiles are numbered
// (ty * ntx + tx) * nz + z; order 0 visits them in that order (z fastest),
// order 1 x fastest.
__device__ __forceinline__ int tile_of(int k, int order, int nz, int ntx, int nty) {
  if (order == 0) return k;
  const int tx = k % ntx, rest = k / ntx;
  const int ty = rest % nty, z = rest / nty;
  return (ty * ntx + tx) * nz + z;
}


// Fused LK iteration (utils/calFlow3d_Wei_v1.py:442-588).
//
// Persistent CTAs take (z slice, window or leftover tile) tiles in turn.  For
// each tile, phase 1 takes every voxel of the tile plus a one-voxel halo as
// independent work: the motion from the tile's CP factors (shared memory),
// the warped moving level and its gradients from one set of 8 float4 corners
// (m, Gx, Gy, Gz share the trilinear weights), It_raw = ref - warped, and for
// tile voxels the clipped gradients and the exclusion mask.  Phase 2 smooths It with the 3x3
// box (edge-replicated), applies the mask and accumulates It^2 and the nine
// gradient products; a window hanging over the volume edge counts the edge
// voxel once per replicated position (mode="nearest" of
// utils/calculate.py:51).  Sums are reduced with warp shuffles in a fixed
// order, so results are deterministic.
//
// DIFF0 != kNoDiff (the launch after a level's first update, MODE = CP): the
// kernel also takes max |motion - initial field| over the tile voxels, where
// the initial field (DIFF0 = UP / DENSE / ZERO) is not a function of this
// level's CPs (utils/calFlow3d_Wei_v1.py:641-643), into st->maxdiff_bits.
template <int MODE, int DIFF0, bool MASK, int PREC, int ORDER>
__global__ void __launch_bounds__(kAccThreads, 4) k_lk_accumulate(IterArgs a) {
  typedef Store<PREC> S;
  // a level that has stopped leaves its remaining iteration launches empty
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
  // persistent CTAs take tiles in turn
  for (int k = blockIdx.x; k < ntiles; k += gridDim.x) {
    const int tile = ORDER ? tile_of(k, ORDER, nz, a.ntx, a.nty) : k;
#include "wr_acc_tile.inc"
  }
  if (DIFF0 != kNoDiff) {
    const float mx = block_max(dmax, red);
    if (threadIdx.x == 0 && mx > 0.f) atomicMax(&a.st->maxdiff_bits, __float_as_uint(mx));
  }
}

// ---------------------------------------------------------------------------
// error evaluation and stopping rules (utils/calFlow3d_Wei_v1.py:101-131,501-530)
// ---------------------------------------------------------------------------

// F32HIST: the error history is a float32 array compared with the new
// error as NumPy does for a Python float (cast to float32 first), the
// cross-resolution rule (utils/calFlowCrossResolution.py:2093,2140-2152).
template <bool F32HIST = false>
__device__ __forceinline__ void decide_body(LKState* st, const double* __restrict__ errpart,
                                            const double* __restrict__ penpart, long long nblk, double n_vox,
                                            double sps, int level, int it, int iter, double tol, int forced) {
  if (!st->active) return;
  __shared__ double red[2][1024];
  double e = 0.0, p = 0.0;
  for (long long i = threadIdx.x; i < nblk; i += blockDim.x) {
    e += errpart[i];
    p += penpart[i];
  }
  red[0][threadIdx.x] = e;
  red[1][threadIdx.x] = p;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[0][threadIdx.x] += red[0][threadIdx.x + s];
      red[1][threadIdx.x] += red[1][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double diff = red[0][0] / n_vox;
  const double pen = red[1][0] * sps / n_vox;
  const double cur = diff + pen;
  WrLKStats& S = st->stats;
  const int e_idx = S.evals[level];
  if (e_idx < WR_MAX_ITERS) {
    S.diff_error[level][e_idx] = diff;
    S.penalty_error[level][e_idx] = pen;
  }
  S.evals[level] = e_idx + 1;
  S.current_error = cur;
  bool stop;
  if (forced >= 0) {
    stop = st->n_updates >= forced;
  } else if (it == iter - 1) {
    stop = true;
  } else {
    if (F32HIST) {
      const float cf = (float)cur;
      const int n_le = ((float)st->old_err[0] <= cf) + ((float)st->old_err[1] <= cf) + ((float)st->old_err[2] <= cf);
      if (n_le > 1) stop = true;
      else if (fabsf(__fsub_rn((float)st->old_err[2], cf)) < (float)tol) stop = true;
      else stop = false;
    } else {
      const int n_le = (st->old_err[0] <= cur) + (st->old_err[1] <= cur) + (st->old_err[2] <= cur);
      if (n_le > 1) stop = true;
      else if (fabs(st->old_err[2] - cur) < tol) stop = true;
      else stop = false;
    }
    if (!stop) {
      st->old_err[0] = st->old_err[1];
      st->old_err[1] = st->old_err[2];
      st->old_err[2] = F32HIST ? (double)(float)cur : cur;
    }
  }
  if (stop) {
    st->active = 0;
    st->do_update = 0;
  } else {
    st->do_update = 1;
  }
}

__global__ void k_decide(LKState* st, const double* __restrict__ errpart, const double* __restrict__ penpart,
                         long long nblk, double n_vox, double sps, int level, int it, int iter, double tol,
                         int forced) {
  decide_body(st, errpart, penpart, nblk, n_vox, sps, level, it, iter, tol, forced);
}

__global__ void k_decide_f32hist(LKState* st, const double* __restrict__ errpart, const double* __restrict__ penpart,
                                 long long nblk, double n_vox, double sps, int level, int it, int iter, double tol,
                                 int forced) {
  decide_body<true>(st, errpart, penpart, nblk, n_vox, sps, level, it, iter, tol, forced);
}

// ---------------------------------------------------------------------------
// CP solve and update (utils/calFlow3d_Wei_v1.py:209-262,591-624)
// ---------------------------------------------------------------------------

// Regularised 3x3 solve by adjugate / determinant: float64 (the reference's
// arithmetic) or float32 re-solved in float64 when the Frobenius condition
// estimate |A| |adj A| / |det A| exceeds 1e6 or the float32 result is not finite.
template <typename R>
__device__ __forceinline__ void solve3(R ixx, R ixy, R ixz, R iyy, R iyz, R izz, R ixt, R iyt, R izt, R& vx, R& vy,
                                       R& vz, R& cond) {
  const R det = ixx * (iyy * izz - iyz * iyz) - ixy * (ixy * izz - iyz * ixz) + ixz * (ixy * iyz - iyy * ixz);
  const R m11 = iyy * izz - iyz * iyz;
  const R m12 = -(ixy * izz - iyz * ixz);
  const R m13 = ixy * iyz - iyy * ixz;
  const R m22 = ixx * izz - ixz * ixz;
  const R m23 = -(ixx * iyz - ixy * ixz);
  const R m33 = ixx * iyy - ixy * ixy;
  vx = (m11 * ixt + m12 * iyt + m13 * izt) / det;
  vy = (m12 * ixt + m22 * iyt + m23 * izt) / det;
  vz = (m13 * ixt + m23 * iyt + m33 * izt) / det;
  const R na = ixx * ixx + iyy * iyy + izz * izz + R(2) * (ixy * ixy + ixz * ixz + iyz * iyz);
  const R nb = m11 * m11 + m22 * m22 + m33 * m33 + R(2) * (m12 * m12 + m13 * m13 + m23 * m23);
  cond = sqrt(na * nb) / fabs(det);
}

// CP i of one item (all threads of the block call it; i >= ncp contributes nothing)
template <bool MIXED>
__device__ __forceinline__ void update_body(LKState* st, float4* cp, const float* __restrict__ sums, long long ncp,
                                            long long i, double sps, float sps_f, double mov_range,
                                            double zratio_d) {
  if (!st->do_update) return;
  __shared__ float red[64];
  float dmax = 0.f;
  int nan_count = 0, fp64_count = 0;
  if (i < ncp) {
    const float* s = sums + i * 12;
    const float ntx = __fmul_rn(sps_f, s[9]), nty = __fmul_rn(sps_f, s[10]), ntz = __fmul_rn(sps_f, s[11]);
    double vx, vy, vz;
    bool done = false;
    if (MIXED) {
      const float fs = (float)sps;
      float fx, fy, fz, fc;
      solve3<float>(s[0] + fs, s[1], s[2], s[3] + fs, s[4], s[5] + fs, s[6] + ntx, s[7] + nty, s[8] + ntz, fx, fy, fz, fc);
      if (isfinite(fx) && isfinite(fy) && isfinite(fz) && fc <= 1e6f) {
        vx = fx; vy = fy; vz = fz;
        done = true;
      } else {
        ++fp64_count;
      }
    }
    if (!done) {
      double dc;
      solve3<double>((double)s[0] + sps, s[1], s[2], (double)s[3] + sps, s[4], (double)s[5] + sps,
                     (double)s[6] + (double)ntx, (double)s[7] + (double)nty, (double)s[8] + (double)ntz, vx, vy, vz, dc);
    }
    if (isnan(vx)) { vx = 0.0; ++nan_count; }
    if (isnan(vy)) { vy = 0.0; ++nan_count; }
    if (isnan(vz)) { vz = 0.0; ++nan_count; }
    double dist = sqrt(vx * vx + vy * vy + vz * vz);
    dist = fmax(dist / mov_range, 1.0);
    vx /= dist;
    vy /= dist;
    vz = (vz / dist) / zratio_d;
    const float4 old = cp[i];
    const float nx = (float)((double)old.x + vx);
    const float ny = (float)((double)old.y + vy);
    const float nz = (float)((double)old.z + vz);
    cp[i] = make_float4(nx, ny, nz, 0.f);
    dmax = fmaxf(fmaxf(fabsf(nx - old.x), fabsf(ny - old.y)), fabsf(nz - old.z));
  }
  if (nan_count) atomicAdd(&st->stats.nan_solves, nan_count);
  if (fp64_count) atomicAdd(&st->stats.fp64_solves, fp64_count);
  const float m = block_max(dmax, red);
  if (threadIdx.x == 0 && m > 0.f) atomicMax(&st->maxdiff_bits, __float_as_uint(m));
}

template <bool MIXED>
__global__ void __launch_bounds__(kThreads) k_update(LKState* st, float4* cp, const float* __restrict__ sums,
                                                    long long ncp, double sps, float sps_f, double mov_range,
                                                    double zratio_d) {
  update_body<MIXED>(st, cp, sums, ncp, blockIdx.x * (long long)blockDim.x + threadIdx.x, sps, sps_f, mov_range,
                     zratio_d);
}


// getMotion stops a level once an update moves no voxel by 1e-3 or more
// (utils/calFlow3d_Wei_v1.py:641-654); the float32 maximum compared with the
// float32 threshold gives the same decisions as the float64 comparison.
constexpr float kMotionTol = 1e-3f;

// after an update: log max |delta motion| and stop the level when it is below
// md_tol (kMotionTol for getMotion, tol for the cross-resolution path)
// (utils/calFlow3d_Wei_v1.py:641-654).  defer: the level's first update,
// whose max over the voxels the next iteration's launch completes
// (k_first_post).
__device__ __forceinline__ void k_post_body(LKState* st, int level, int forced, int defer, float md_tol) {
  if (!st->do_update) return;
  WrLKStats& S = st->stats;
  // the level's log runs on across passes (the cross-resolution correction
  // re-runs a level): its slot is the level's update count, not this pass's
  const int slot = S.updates[level];
  st->n_updates += 1;
  S.updates[level] = slot + 1;
  st->do_update = 0;
  if (defer) return;
  const float md = __uint_as_float(st->maxdiff_bits);
  if (slot < WR_MAX_ITERS) S.max_diff_motion[level][slot] = (double)md;
  if (forced < 0 && md < md_tol) st->active = 0;
  st->maxdiff_bits = 0u;
}

__global__ void k_post(LKState* st, int level, int forced, int defer, float md_tol) {
  k_post_body(st, level, forced, defer, md_tol);
}

// The level's first update, once the following launch has added max
// |new - initial| over the voxels: log it and apply the md_tol rule.  A level
// that stops here discards that launch's error and sums (k_decide and
// k_update skip an inactive level).
__device__ __forceinline__ void k_first_post_body(LKState* st, int level, int forced, float md_tol) {
  if (!st->active) return;
  const float md = __uint_as_float(st->maxdiff_bits);
  const int slot = st->stats.updates[level] - 1;   // this pass's first update
  if (slot >= 0 && slot < WR_MAX_ITERS) st->stats.max_diff_motion[level][slot] = (double)md;
  if (forced < 0 && md < md_tol) st->active = 0;
  st->maxdiff_bits = 0u;
}

__global__ void k_first_post(LKState* st, int level, int forced, float md_tol) {
  k_first_post_body(st, level, forced, md_tol);
}

// ---------------------------------------------------------------------------
// batched registration: the frames of a batch (shapes may differ) advance
// through the levels together, one launch per kernel for the whole batch;
// each frame keeps its own stopping state, so frames whose level has
// stopped simply contribute no work.
// ---------------------------------------------------------------------------

constexpr int kMaxBatch = WR_MAX_BATCH;

struct BatchIter {             // one batched launch of the fused iteration
  int n, order;
  int tile_start[kMaxBatch + 1];   // prefix sums of the frames' tile counts
  IterArgs item[kMaxBatch];
};

__device__ __forceinline__ void flush_max(float& dmax, LKState* st, float* red) {
  const float mx = block_max(dmax, red);
  if (threadIdx.x == 0 && mx > 0.f) atomicMax(&st->maxdiff_bits, __float_as_uint(mx));
  dmax = 0.f;
}

template <int MODE, int DIFF0, bool MASK, int PREC>
__global__ void __launch_bounds__(kAccThreads, 4) k_lk_accumulate_batch(const __grid_constant__ BatchIter b) {
  typedef Store<PREC> S;
  extern __shared__ float4 smem4[];
  float dmax = 0.f;
  int cur = 0;
  for (int k = blockIdx.x; k < b.tile_start[b.n]; k += gridDim.x) {
    int i = cur;
    while (k >= b.tile_start[i + 1]) ++i;
    if (i != cur) {
      // the start of shared memory is free between tiles (the tail's barrier)
      if (DIFF0 != kNoDiff) flush_max(dmax, b.item[cur].st, reinterpret_cast<float*>(smem4));
      cur = i;
    }
    const IterArgs& a = b.item[i];
    if (!*(volatile const int*)&a.st->active) continue;
    const int nx = a.mov.nx, ny = a.mov.ny, nz = a.mov.nz;
    const int w = a.w;
    // frames may differ in patch width: the carve-up follows the tile's frame
    // (the launch's dynamic shared memory covers the widest)
    const AccSmem sm(smem4, w);
    float4* gsm = sm.gsm;
    float* it_raw = sm.it_raw;
    const TileField tf = sm.tf;
    int* flags = sm.flags;
    float* red = sm.red;
    const TileField tf0 = sm.tf0;
    int* flags0 = sm.flags0;
    const int ncx = a.cpv.ncx, ncy = a.cpv.ncy;
    const int tile = tile_of(k - b.tile_start[i], b.order, nz, a.ntx, a.nty);
#include "wr_acc_tile.inc"
  }
  if (DIFF0 != kNoDiff) flush_max(dmax, b.item[cur].st, reinterpret_cast<float*>(smem4));
}

struct BatchDecide {
  int n;
  LKState* st[kMaxBatch];
  const double* errpart[kMaxBatch];
  const double* penpart[kMaxBatch];
  long long nblk[kMaxBatch];
  double n_vox[kMaxBatch];
  double sps[kMaxBatch];        // smoothPenalty x (2r + 1)^2 of each frame
  double tol[kMaxBatch];
  int iter[kMaxBatch];
  int forced[kMaxBatch];
};

// one block per frame
__global__ void k_decide_batch(const __grid_constant__ BatchDecide b, int level, int it) {
  const int i = blockIdx.x;
  decide_body(b.st[i], b.errpart[i], b.penpart[i], b.nblk[i], b.n_vox[i], b.sps[i], level, it, b.iter[i], b.tol[i],
              b.forced[i]);
}

struct BatchUpdate {
  int n;
  LKState* st[kMaxBatch];
  float4* cp[kMaxBatch];
  const float* sums[kMaxBatch];
  long long ncp[kMaxBatch];
  double sps[kMaxBatch];
  float sps_f[kMaxBatch];
  double mov_range[kMaxBatch];
  double zratio_d[kMaxBatch];   // the level's zRatio of each frame
};

// blockIdx.y = frame
template <bool MIXED>
__global__ void __launch_bounds__(kThreads) k_update_batch(const __grid_constant__ BatchUpdate b) {
  const int f = blockIdx.y;
  update_body<MIXED>(b.st[f], b.cp[f], b.sums[f], b.ncp[f], blockIdx.x * (long long)blockDim.x + threadIdx.x, b.sps[f],
                     b.sps_f[f], b.mov_range[f], b.zratio_d[f]);
}

struct BatchState {
  int n;
  LKState* st[kMaxBatch];
  int forced[kMaxBatch];
};

// one thread per frame
__global__ void k_post_batch(const __grid_constant__ BatchState b, int level, int defer) {
  if (threadIdx.x < b.n) k_post_body(b.st[threadIdx.x], level, b.forced[threadIdx.x], defer, kMotionTol);
}

__global__ void k_first_post_batch(const __grid_constant__ BatchState b, int level) {
  if (threadIdx.x < b.n) k_first_post_body(b.st[threadIdx.x], level, b.forced[threadIdx.x], kMotionTol);
}

__global__ void k_level_begin(LKState* st, int level, int first) {
  if (first) {
    WrLKStats z = {};
    st->stats = z;
  }
  st->active = 1;
  st->do_update = 0;
  st->level = level;
  st->n_updates = 0;
  st->maxdiff_bits = 0u;
  st->old_err[0] = st->old_err[1] = st->old_err[2] = INFINITY;
  st->stats.evals[level] = 0;
  st->stats.updates[level] = 0;
}

// motion_current at the CP voxels at a level's start
template <int MODE0>
__global__ void k_cp_init(float4* cp, FieldSrc f, int ncx, int ncy, int nz, int r, int w) {
  const long long n = (long long)ncx * ncy * nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int cx = (int)(i % ncx);
    const long long rest = i / ncx;
    const int cy = (int)(rest % ncy);
    const int z = (int)(rest / ncy);
    const float3 v = eval_field<MODE0>(f, r + cx * w, r + cy * w, z);
    cp[i] = make_float4(v.x, v.y, v.z, 0.f);
  }
}

// dense field of a level from a field source (used when no update can occur
// at some level, and for the coarsest level's initial field)
template <int MODE0>
__global__ void k_dense_from(float4* out, FieldSrc f, int nx, int ny, int nz) {
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    WR_FOR_COLS(nx, x) {
      const float3 v = eval_field<MODE0>(f, x, y, z);
      out[(size_t)row * nx + x] = make_float4(v.x, v.y, v.z, 0.f);
    }
  }
}

// coarsest-level initial field from option["motion"] resized per component,
// divided by the full-res/level size ratio (utils/calFlow3d_Wei_v1.py:362-377)
__global__ void k_dense_init_pack(float4* out, const float* c0, const float* c1, const float* c2, long long n,
                                  double dx, double dy, double dz) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = make_float4((float)((double)c0[i] / dx), (float)((double)c1[i] / dy), (float)((double)c2[i] / dz), 0.f);
}

// final motion (z, y, x, 3)
// getMotion's error_log snapshot of one iteration (utils/calFlow3d_Wei_v1.py:
// 451-470): the level's dense motion (z, y, x, 3) and the moving level warped
// by it (trilinear, taps clamped to the level); nothing when the level has
// stopped before this iteration.
template <int MODE, int PREC>
__global__ void k_snapshot(const LKState* st, FieldSrc f, const typename Store<PREC>::V4* __restrict__ movg, int nx,
                           int ny, int nz, float* __restrict__ motion, float* __restrict__ warped) {
  typedef Store<PREC> S;
  if (!*(volatile const int*)&st->active) return;
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    WR_FOR_COLS(nx, x) {
      const float3 m = eval_field<MODE>(f, x, y, z);
      const size_t i = ((size_t)z * ny + y) * nx + x;
      if (motion) {
        motion[3 * i] = m.x;
        motion[3 * i + 1] = m.y;
        motion[3 * i + 2] = m.z;
      }
      if (warped) {
        int x0, y0, z0;
        float tx, ty, tz;
        split_coord((float)x + m.x, x0, tx);
        split_coord((float)y + m.y, y0, ty);
        split_coord((float)z + m.z, z0, tz);
        const int xs[2] = {clampi(x0, 0, nx - 1), clampi(x0 + 1, 0, nx - 1)};
        const int ys[2] = {clampi(y0, 0, ny - 1), clampi(y0 + 1, 0, ny - 1)};
        const int zs[2] = {clampi(z0, 0, nz - 1), clampi(z0 + 1, 0, nz - 1)};
        float acc = 0.f;
        for (int c = 0; c < 2; ++c)
          for (int b = 0; b < 2; ++b)
            for (int a = 0; a < 2; ++a) {
              const float wgt = (a ? tx : 1.f - tx) * (b ? ty : 1.f - ty) * (c ? tz : 1.f - tz);
              acc = fmaf(wgt, S::load_m(movg + ((size_t)zs[c] * ny + ys[b]) * nx + xs[a]), acc);
            }
        warped[i] = acc;
      }
    }
  }
}

// a level's reference and moving images as float32 (error_log "data_ref" / "data_mov")
template <int PREC>
__global__ void k_level_images(const typename Store<PREC>::V1* __restrict__ ref,
                               const typename Store<PREC>::V4* __restrict__ movg, long long n, float* ref_out,
                               float* mov_out) {
  typedef Store<PREC> S;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (ref_out) ref_out[i] = S::load1(ref + i);
    if (mov_out) mov_out[i] = S::load_m(movg + i);
  }
}

template <int MODE>
__global__ void k_write_motion(float* __restrict__ out, FieldSrc f, int nx, int ny, int nz) {
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    float* o = out + (size_t)row * nx * 3;
    WR_FOR_COLS(nx, x) {
      const float3 v = eval_field<MODE>(f, x, y, z);
      o[3 * x + 0] = v.x;
      o[3 * x + 1] = v.y;
      o[3 * x + 2] = v.z;
    }
  }
}

// ---------------------------------------------------------------------------
// correctMotion (utils/calFlow3d_Wei_v1.py:676-706): pull warp, float64
// trilinear arithmetic on float32 values, float32 result
// ---------------------------------------------------------------------------

// src sampled at (x, y, z) + m: float64 trilinear weights on the (clamped)
// float32 corner values, rounded once to float32.
template <typename T>
__device__ __forceinline__ float warp_sample(const T* __restrict__ src, int nx, int ny, int nz, int x, int y, int z,
                                             float mx, float my, float mz) {
  const size_t sy = nx, sz = (size_t)nx * ny;
  const float cx = (float)x + mx, cy = (float)y + my, cz = (float)z + mz;
  int x0, y0, z0;
  float tx_f, ty_f, tz_f;
  split_coord(cx, x0, tx_f);
  split_coord(cy, y0, ty_f);
  split_coord(cz, z0, tz_f);
  const double tx = tx_f, ty = ty_f, tz = tz_f;
  const int xa = clampi(x0, 0, nx - 1), xb = clampi(x0 + 1, 0, nx - 1);
  const int ya = clampi(y0, 0, ny - 1), yb = clampi(y0 + 1, 0, ny - 1);
  const int za = clampi(z0, 0, nz - 1), zb = clampi(z0 + 1, 0, nz - 1);
  // one base address and the three tap offsets (0 where a tap is clamped)
  const T* p = src + (za * sz + ya * sy + xa);
  const size_t ox = (size_t)(xb - xa), oy = (size_t)(yb - ya) * sy, oz = (size_t)(zb - za) * sz;
  const double c000 = load_f<T>(p, 0), c001 = load_f<T>(p, ox);
  const double c010 = load_f<T>(p, oy), c011 = load_f<T>(p, oy + ox);
  const double c100 = load_f<T>(p, oz), c101 = load_f<T>(p, oz + ox);
  const double c110 = load_f<T>(p, oz + oy), c111 = load_f<T>(p, oz + oy + ox);
  const double wx0 = 1.0 - tx, wy0 = 1.0 - ty, wz0 = 1.0 - tz;
  const double v = wx0 * wy0 * wz0 * c000 + tx * wy0 * wz0 * c001 + wx0 * ty * wz0 * c010 + tx * ty * wz0 * c011 +
                   wx0 * wy0 * tz * c100 + tx * wy0 * tz * c101 + wx0 * ty * tz * c110 + tx * ty * tz * c111;
  return (float)v;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_warp(const T* __restrict__ src, const float* __restrict__ motion,
                                                  float* __restrict__ out, int nz, int ny, int nx) {
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    const float* mrow = motion + (size_t)row * nx * 3;
    WR_FOR_COLS(nx, x) {
      out[(size_t)row * nx + x] = warp_sample<T>(src, nx, ny, nz, x, y, z, __ldg(mrow + 3 * x + 0),
                                                 __ldg(mrow + 3 * x + 1), __ldg(mrow + 3 * x + 2));
    }
  }
}

// final motion (z, y, x, 3) and mov warped by it (correctMotion) in one pass:
// the same values as k_write_motion followed by k_warp
template <int MODE, typename T>
__global__ void __launch_bounds__(kThreads) k_write_motion_warp(float* __restrict__ out, float* __restrict__ warped,
                                                               const T* __restrict__ src, FieldSrc f, int nx, int ny,
                                                               int nz) {
  WR_FOR_ROWS(nz * ny, row) {
    const int z = row / ny, y = row - z * ny;
    float* o = out + (size_t)row * nx * 3;
    WR_FOR_COLS(nx, x) {
      const float3 v = eval_field<MODE>(f, x, y, z);
      o[3 * x + 0] = v.x;
      o[3 * x + 1] = v.y;
      o[3 * x + 2] = v.z;
      warped[(size_t)row * nx + x] = warp_sample<T>(src, nx, ny, nz, x, y, z, v.x, v.y, v.z);
    }
  }
}

// ---------------------------------------------------------------------------
// smoothness-penalty normalisation factor (utils/preprocess.py:42-66)
// ---------------------------------------------------------------------------

template <typename T>
__global__ void __launch_bounds__(kThreads) k_penalty_partial(const T* __restrict__ ref, const uint8_t* __restrict__ excl,
                                                             double* __restrict__ part, int nz, int ny, int nx) {
  __shared__ double red[4][kThreads];
  const long long n = (long long)nx * ny * nz;
  double sxx = 0.0, syy = 0.0, cx = 0.0, cy = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const long long rest = i / nx;
    const int y = (int)(rest % ny);
    const bool keep = excl == nullptr || excl[i] == 0;
    if (!keep) continue;
    if (x >= 1 && x <= nx - 2) {
      const double d = ((double)load_f<T>(ref, i + 1) - (double)load_f<T>(ref, i - 1)) / 2.0;
      sxx += d * d;
      cx += 1.0;
    }
    if (y >= 1 && y <= ny - 2) {
      const double d = ((double)load_f<T>(ref, i + nx) - (double)load_f<T>(ref, i - nx)) / 2.0;
      syy += d * d;
      cy += 1.0;
    }
  }
  red[0][threadIdx.x] = sxx;
  red[1][threadIdx.x] = syy;
  red[2][threadIdx.x] = cx;
  red[3][threadIdx.x] = cy;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 4) part[4 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_penalty_final(const double* __restrict__ part, int nblk, double* out) {
  __shared__ double red[4][1024];
  double v[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x)
    for (int k = 0; k < 4; ++k) v[k] += part[4 * b + k];
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = (red[0][0] / red[2][0] + red[1][0] / red[3][0]) / 2.0;
}

}  // namespace wr
