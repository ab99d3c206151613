// C ABI of the B200 registration path: planning, workspace layout and the
// launch sequence that replaces getMotion / correctMotion
// (utils/calFlow3d_Wei_v1.py:295-706 of the reference package).
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "wr_b200.h"
#include "wr_kernels.cuh"
#include "wr_plan.h"
#include "wr_xres.cuh"
#include "wr_xres_wr.cuh"
#include "wr_xres.h"
#include <cmath>
#include <algorithm>
#include <cub/cub.cuh>

namespace wr {

static thread_local std::string g_last_error;

static int fail(int code, const char* msg) {
  g_last_error = msg ? msg : "";
  return code;
}

static int cuda_fail(cudaError_t e, const char* where) {
  g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
  return -(int)e;
}

static size_t align_up(size_t v, size_t a = 256) { return (v + a - 1) / a * a; }

struct Alloc {
  size_t cur = 0;
  size_t take(size_t bytes) {
    size_t off = cur;
    cur = align_up(cur + bytes);
    return off;
  }
};

// Shift-invariant interior of the full-res -> level table along one axis:
// the widest range of outputs around the middle whose tap rows (as
// resize_row computes them) read in[s*o + c0 + t] with bit-identical weights.
static SITaps find_si_taps(int in_len, int out_len) {
  SITaps si;
  memset(&si, 0, sizeof(si));
  const int P = resize_taps(in_len, out_len);
  if (P > kSIMaxTaps || out_len < 1 || in_len % out_len != 0) return si;
  const int s = in_len / out_len;
  std::vector<double> w((size_t)out_len * P);
  std::vector<int32_t> ix((size_t)out_len * P);
  for (int k = 0; k < out_len; ++k) resize_row(in_len, out_len, RESIZE_BICUBIC, k, &w[(size_t)k * P], &ix[(size_t)k * P]);
  const int mid = out_len / 2;
  const int c0 = ix[(size_t)mid * P] - s * mid;
  auto fits = [&](int k) {
    for (int t = 0; t < P; ++t) {
      if (ix[(size_t)k * P + t] != s * k + c0 + t) return false;
      if (memcmp(&w[(size_t)k * P + t], &w[(size_t)mid * P + t], sizeof(double)) != 0) return false;
    }
    return true;
  };
  if (!fits(mid)) return si;
  int lo = mid, hi = mid + 1;
  while (lo > 0 && fits(lo - 1)) --lo;
  while (hi < out_len && fits(hi)) ++hi;
  si.P = P; si.s = s; si.c0 = c0; si.lo = lo; si.hi = hi;
  si.ls = in_len / s + 1;
  volatile double acc = 0.0;   // tap-order float64 sum, no contraction
  for (int t = 0; t < P; ++t) acc = acc + w[(size_t)mid * P + t];
  si.wsum = acc;
  for (int t = 0; t < P; ++t) {
    si.w[t] = w[(size_t)mid * P + t];
    si.wf[t] = (float)si.w[t];
    const int e = c0 + t;                         // tap position of output 0
    const int q = e >= 0 ? e / s : -((-e + s - 1) / s);
    si.off[t] = (e - q * s) * si.ls + q;
  }
  return si;
}

static int level_extent(int n, int layer) { return (int)((double)n / (double)(1 << layer)); }

// number of k >= 0 with r + k(2r+1) < n - 1 (utils/calFlow3d_Wei_v1.py:434-435)
static int cp_count(int n, int r, int w) {
  int span = n - 1 - r;
  return span > 0 ? (span + w - 1) / w : 0;
}

int make_plan(int nz, int ny, int nx, const WrLKParams* p, bool has_mref, bool has_mmov, bool has_init,
              Plan* plan, const char** why) {
  *why = "";
  if (nz < 1 || ny < 1 || nx < 1) { *why = "volume extents must be positive"; return WR_E_SHAPE; }
  if ((long long)nz * ny * nx > (1LL << 36)) { *why = "volume too large"; return WR_E_SHAPE; }
  if (p->layer < 0 || p->layer >= WR_MAX_LEVELS) { *why = "layer out of range [0, 7]"; return WR_E_PARAM; }
  if (p->iter < 1 || p->iter > WR_MAX_ITERS) { *why = "iter out of range [1, 64]"; return WR_E_PARAM; }
  if (p->r < 1 || p->r > 48) { *why = "r out of range [1, 48]"; return WR_E_PARAM; }
  if (!(p->zRatio > 0.f) || !(p->movRange > 0.f)) { *why = "zRatio and movRange must be positive"; return WR_E_PARAM; }
  if (!(p->smoothPenalty >= 0.0) || !(p->tol >= 0.0)) { *why = "smoothPenalty and tol must be >= 0"; return WR_E_PARAM; }
  if (p->precision != WR_PREC_F32 && p->precision != WR_PREC_F16 && p->precision != WR_PREC_BF16) {
    *why = "precision must be WR_PREC_F32, WR_PREC_F16 or WR_PREC_BF16";
    return WR_E_PARAM;
  }
  Plan& P = *plan;
  memset(&P, 0, sizeof(P));
  P.nz = nz; P.ny = ny; P.nx = nx;
  P.levels = p->layer + 1;
  P.r = p->r; P.w = 2 * p->r + 1; P.iter = p->iter;
  P.has_mref = has_mref; P.has_mmov = has_mmov; P.has_init = has_init;
  P.dense_all = p->iter == 1;
  for (int l = 0; l < P.levels; ++l) P.dense_out[l] = P.dense_all || p->forced_updates[l] == 0;
  for (int l = 0; l < P.levels; ++l) P.dense_in[l] = P.dense_out[l] || (l + 1 < P.levels && P.dense_out[l + 1]);
  P.precision = p->precision;
  Alloc A;
  size_t tmp_a = 0, tmp_b = 0;
  for (int l = 0; l < P.levels; ++l) {
    LevelPlan& L = P.lv[l];
    L.nx = level_extent(nx, l);
    L.ny = level_extent(ny, l);
    L.nz = nz;
    if (L.nx < 1 || L.ny < 1) { *why = "volume too small for this many pyramid levels"; return WR_E_SHAPE; }
    L.ncx = cp_count(L.nx, P.r, P.w);
    L.ncy = cp_count(L.ny, P.r, P.w);
    if (L.ncx < 1 || L.ncy < 1) { *why = "a pyramid level has no control point (volume too small for r)"; return WR_E_NOCP; }
    // implied by the line above for r >= 1; the iteration kernel's tap pairs rely on it
    if (L.nx < 3 || L.ny < 3) { *why = "a pyramid level is narrower than 3 voxels"; return WR_E_NOCP; }
    L.ntx = L.ncx + (L.nx > L.ncx * P.w ? 1 : 0);
    L.nty = L.ncy + (L.ny > L.ncy * P.w ? 1 : 0);
    L.n = (long long)L.nx * L.ny * L.nz;
    if (L.n >= (1LL << 31)) { *why = "a pyramid level holds 2^31 voxels or more"; return WR_E_SHAPE; }
    L.ncp = (long long)L.ncx * L.ncy * L.nz;
    L.nblk = (long long)L.ntx * L.nty * L.nz;
    L.zratio_d = (double)p->zRatio / (double)(1 << l);
    L.zratio = (float)L.zratio_d;
    double sx = resize_scale(nx, L.nx), sy = resize_scale(ny, L.ny);
    L.x_first = sx <= sy;
    L.tx_taps = resize_taps(nx, L.nx);
    L.ty_taps = resize_taps(ny, L.ny);
    if (l > 0) {
      L.six = find_si_taps(nx, L.nx);
      L.siy = find_si_taps(ny, L.ny);
    }
    const size_t vbytes = p->precision == WR_PREC_F32 ? 4 : 2;   // per stored channel value
    L.ref = A.take((size_t)L.n * vbytes);
    L.movg = A.take((size_t)L.n * 4 * vbytes);
    L.mbits = A.take((size_t)L.n);
    L.mmov = A.take((size_t)L.n * 4);
    L.cp = A.take((size_t)L.ncp * 16);
    L.sums = A.take((size_t)L.ncp * 12 * 4);
    L.errpart = A.take((size_t)L.nblk * 8);
    L.penpart = A.take((size_t)L.nblk * 8);
    L.dense = (P.dense_in[l] || l == P.levels - 1) ? A.take((size_t)L.n * 16) : 0;
    L.tx_w = A.take((size_t)L.nx * L.tx_taps * 8);
    L.tx_i = A.take((size_t)L.nx * L.tx_taps * 4);
    L.ty_w = A.take((size_t)L.ny * L.ty_taps * 8);
    L.ty_i = A.take((size_t)L.ny * L.ty_taps * 4);
    L.ux_w = A.take((size_t)L.nx * 2 * 4);
    L.ux_i = A.take((size_t)L.nx * 2 * 4);
    L.uy_w = A.take((size_t)L.ny * 2 * 4);
    L.uy_i = A.take((size_t)L.ny * 2 * 4);
    if (l > 0) {
      size_t first = L.x_first ? (size_t)nz * ny * L.nx : (size_t)nz * L.ny * nx;
      tmp_a = first > tmp_a ? first : tmp_a;
      tmp_b = (size_t)L.n > tmp_b ? (size_t)L.n : tmp_b;
    }
  }
  for (int l = 0; l + 1 < P.levels; ++l) {
    double sx = resize_scale(P.lv[l + 1].nx, P.lv[l].nx), sy = resize_scale(P.lv[l + 1].ny, P.lv[l].ny);
    P.lv[l].up_x_first = sx <= sy;
  }
  {
    // the initial-field resize of the coarsest level reuses the temporaries
    const LevelPlan& C = P.lv[P.levels - 1];
    size_t first = C.x_first ? (size_t)nz * ny * C.nx : (size_t)nz * C.ny * nx;
    tmp_a = first > tmp_a ? first : tmp_a;
    tmp_b = (size_t)C.n * 3 > tmp_b ? (size_t)C.n * 3 : tmp_b;
  }
  // row-major x tables before their transpose
  size_t tab = 0;
  for (int l = 0; l < P.levels; ++l) {
    const size_t b = (size_t)P.lv[l].nx * P.lv[l].tx_taps * 12;
    tab = b > tab ? b : tab;
  }
  P.tab_scratch = A.take(tab);
  P.tmp_a_bytes = tmp_a * 8;
  P.tmp_b_bytes = tmp_b * 8;
  P.tmp_a = A.take(P.tmp_a_bytes);
  P.tmp_b = A.take(P.tmp_b_bytes);
  P.state = A.take(sizeof(LKState) + 64);
  P.total = A.cur;
  return WR_OK;
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------

static int grid_for(long long n, int threads = kThreads) {
  long long b = (n + threads - 1) / threads;
  long long cap = 148LL * 16;
  if (b < 1) b = 1;
  return (int)(b < cap ? b : cap);
}

// Grid of a row-parallel voxel kernel (blocks of 32 x kRowWarps threads).
static int row_grid(long long nrows) {
  long long b = (nrows + kRowWarps - 1) / kRowWarps;
  long long cap = 148LL * 16;
  if (b < 1) b = 1;
  return (int)(b < cap ? b : cap);
}
static const dim3 kRowBlock(32, kRowWarps);

// null counts as aligned
static bool aligned(const void* p, size_t bytes) { return ((uintptr_t)p % bytes) == 0; }

template <typename T> static T* at_off(void* base, size_t off) {
  return reinterpret_cast<T*>(static_cast<char*>(base) + off);
}


// x pass of a resize: rows staged in shared memory when the table has a
// shift-invariant interior with a down-scale factor of 2, 4 or 8 and the
// staged rows fit, else straight from global memory.
template <int S, typename Tin, typename A, typename Tout>
static bool resample_x_si(const SITaps& si, const Tin* in, Tout* out, int nrows, int nx_in, int nx_out,
                          const double* w, const int32_t* idx, cudaStream_t s) {
  if (si.s != S || si.P != 4 * S + 2) return false;
  size_t smem;
  void (*kern)(const SITaps, const Tin*, Tout*, int, int, int, const double*, const int32_t*);
  if constexpr (std::is_same<Tin, uint8_t>::value && std::is_same<A, double>::value &&
                std::is_same<Tout, double>::value) {
    smem = (size_t)kStageWarps * mask_stage_bytes(nx_in) + mask_edge_bytes<S>();
    kern = k_resample_x_mask<S>;
  } else {
    if (si.c0 == kPPFirstTap<S> && nx_in <= kPPMaxIn && si.lo + (nx_out - si.hi) <= kPPMaxEdge &&
        aligned(in, S * sizeof(Tin))) {
      // rows staged relative to the first tap, static shared memory
      long long g = (nrows + kStageWarps - 1) / kStageWarps;
      if (g > 148LL * 32) g = 148LL * 32;
      k_resample_x_pp<S, Tin, A, Tout><<<(int)g, dim3(32, kStageWarps), 0, s>>>(si, in, out, nrows, nx_in, nx_out,
                                                                             w, idx);
      return true;
    }
    smem = (size_t)kStageWarps * S * si.ls * sizeof(A);
    kern = k_resample_x_si<S, Tin, A, Tout>;
  }
  if (smem > 96 * 1024) return false;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  long long g = (nrows + kStageWarps - 1) / kStageWarps;
  if (g > 148LL * 32) g = 148LL * 32;
  kern<<<(int)g, dim3(32, kStageWarps), smem, s>>>(si, in, out, nrows, nx_in, nx_out, w, idx);
  return true;
}

template <typename Tin, typename A, typename Tout>
static void resample_x(const SITaps& si, const Tin* in, Tout* out, int nrows, int nx_in, int nx_out,
                       const double* w, const int32_t* idx, int P, int stride, int comp, cudaStream_t s) {
  if (si.hi > si.lo && stride == 1 &&
      (resample_x_si<2, Tin, A, Tout>(si, in, out, nrows, nx_in, nx_out, w, idx, s) ||
       resample_x_si<4, Tin, A, Tout>(si, in, out, nrows, nx_in, nx_out, w, idx, s) ||
       resample_x_si<8, Tin, A, Tout>(si, in, out, nrows, nx_in, nx_out, w, idx, s)))
    return;
  k_resample_x<Tin, A, Tout><<<row_grid(nrows), kRowBlock, 0, s>>>(si, in, out, 1, nrows, nx_in, nx_out, w, idx, P,
                                                                   stride, comp);
}

// y pass of a resize: the compile-time-tap kernel for a shift-invariant
// table with a down-scale factor of 2, 4 or 8, else the table kernel.
template <int S, typename Tin, typename A, typename Tout>
static bool resample_y_si(const SITaps& si, const Tin* in, Tout* out, int nz, int ny_in, int ny_out, int nx,
                          const double* w, const int32_t* idx, cudaStream_t s) {
  if (si.s != S || si.P != 4 * S + 2) return false;
  // V adjacent columns per lane: 16-byte loads of float32 / float64 inputs
  constexpr int V = sizeof(Tin) >= 8 ? 2 : 4;
  if (nx % V == 0 && aligned(in, V * sizeof(Tin))) {
    k_resample_y_si_v<S, V, Tin, A, Tout><<<row_grid((long long)nz * ny_out), kRowBlock, 0, s>>>(
        si, in, out, nz, ny_in, ny_out, nx, w, idx);
    return true;
  }
  k_resample_y_si<S, Tin, A, Tout><<<row_grid((long long)nz * ny_out), kRowBlock, 0, s>>>(si, in, out, nz, ny_in,
                                                                                       ny_out, nx, w, idx);
  return true;
}

template <typename Tin, typename A, typename Tout>
static void resample_y(const SITaps& si, const Tin* in, Tout* out, int nz, int ny_in, int ny_out, int nx,
                       const double* w, const int32_t* idx, int P, int stride, int comp, cudaStream_t s) {
  if (si.hi > si.lo && stride == 1 &&
      (resample_y_si<2, Tin, A, Tout>(si, in, out, nz, ny_in, ny_out, nx, w, idx, s) ||
       resample_y_si<4, Tin, A, Tout>(si, in, out, nz, ny_in, ny_out, nx, w, idx, s) ||
       resample_y_si<8, Tin, A, Tout>(si, in, out, nz, ny_in, ny_out, nx, w, idx, s)))
    return;
  k_resample_y<Tin, A, Tout><<<row_grid((long long)nz * ny_out), kRowBlock, 0, s>>>(si, in, out, nz, ny_in, ny_out,
                                                                                    nx, w, idx, P, stride, comp);
}

// Separable resize of a full-resolution volume to a level:
// first pass (x or y, by scale order) into tmp, second pass into `out`.
// A = double with Tin/Tout of any type gives the float64-exact resize.
template <typename Tin, typename A, typename Tout>
static void resize_to_level(const Plan& P, const LevelPlan& L, void* ws, const Tin* in, int stride, int comp,
                            A* tmp, Tout* out, cudaStream_t s) {
  const double* txw = at_off<double>(ws, L.tx_w);
  const int32_t* txi = at_off<int32_t>(ws, L.tx_i);
  const double* tyw = at_off<double>(ws, L.ty_w);
  const int32_t* tyi = at_off<int32_t>(ws, L.ty_i);
  if (L.x_first) {
    resample_x<Tin, A, A>(L.six, in, tmp, P.nz * P.ny, P.nx, L.nx, txw, txi, L.tx_taps, stride, comp, s);
    resample_y<A, A, Tout>(L.siy, tmp, out, P.nz, P.ny, L.ny, L.nx, tyw, tyi, L.ty_taps, 1, 0, s);
  } else {
    resample_y<Tin, A, A>(L.siy, in, tmp, P.nz, P.ny, L.ny, P.nx, tyw, tyi, L.ty_taps, stride, comp, s);
    resample_x<A, A, Tout>(L.six, tmp, out, P.nz * L.ny, P.nx, L.nx, txw, txi, L.tx_taps, 1, 0, s);
  }
}

template <typename T, int PREC>
static void build_pyramid(const Plan& P, void* ws, const T* mov, const T* ref, const uint8_t* mmov_u8,
                          const uint8_t* mref_u8, bool reuse_ref, cudaStream_t s) {
  typedef Store<PREC> S;
  const bool same_mask = mmov_u8 != nullptr && mmov_u8 == mref_u8 && !reuse_ref;
  for (int l = 0; l < P.levels; ++l) {
    const LevelPlan& L = P.lv[l];
    typename S::V1* refl = at_off<typename S::V1>(ws, L.ref);
    typename S::V4* movg = at_off<typename S::V4>(ws, L.movg);
    float* mmov = at_off<float>(ws, L.mmov);
    uint8_t* bits = at_off<uint8_t>(ws, L.mbits);
    const bool any_mask = mmov_u8 || mref_u8;
    if (l == 0) {
      // scale 1 on every axis: the resize is an exact copy
      if (!reuse_ref) k_to_level<T, PREC><<<grid_for(L.n), kThreads, 0, s>>>(ref, refl, L.n);
      // four voxels per lane when rows are a multiple of 4 long and the inputs aligned
      const bool x4 = L.nx % 4 == 0 && aligned(mov, 4 * sizeof(T)) && aligned(mmov_u8, 4) && aligned(mref_u8, 4);
      const int g = row_grid((long long)L.nz * L.ny);
      if (x4) k_pack_movg_x4<T, PREC><<<g, kRowBlock, 0, s>>>(mov, movg, L.nz, L.ny, L.nx);
      else k_pack_movg<T, PREC><<<g, kRowBlock, 0, s>>>(mov, movg, L.nz, L.ny, L.nx);
      // exclusion bits and the moving mask as float, straight from the uint8 masks
      if (any_mask && x4)
        k_mask_bits_u8x4<<<g, kRowBlock, 0, s>>>(reuse_ref ? nullptr : mref_u8, mmov_u8, mmov_u8 ? mmov : nullptr, bits,
                                                 L.nz, L.ny, L.nx, reuse_ref ? 1 : 0);
      else if (any_mask)
        k_mask_bits<uint8_t><<<g, kRowBlock, 0, s>>>(nullptr, reuse_ref ? nullptr : mref_u8, mmov_u8,
                                                     mmov_u8 ? mmov : nullptr, bits, L.nz, L.ny, L.nx,
                                                     reuse_ref ? 1 : 0);
      continue;
    }
    float* tmpf = at_off<float>(ws, P.tmp_a);
    float* levf = at_off<float>(ws, P.tmp_b);
    if (!reuse_ref) {
      if (PREC == WR_PREC_F32) {
        resize_to_level<T, float, float>(P, L, ws, ref, 1, 0, tmpf, reinterpret_cast<float*>(refl), s);
      } else {
        resize_to_level<T, float, float>(P, L, ws, ref, 1, 0, tmpf, levf, s);
        k_store_level<PREC><<<grid_for(L.n), kThreads, 0, s>>>(levf, refl, L.n);
      }
    }
    resize_to_level<T, float, float>(P, L, ws, mov, 1, 0, tmpf, levf, s);
    k_pack_movg<float, PREC><<<row_grid((long long)L.nz * L.ny), kRowBlock, 0, s>>>(levf, movg, L.nz, L.ny, L.nx);
    double* tmpd = at_off<double>(ws, P.tmp_a);
    double* levd = at_off<double>(ws, P.tmp_b);
    if (mmov_u8) {
      if (same_mask) {
        resize_to_level<uint8_t, double, double>(P, L, ws, mmov_u8, 1, 0, tmpd, levd, s);
        k_d_to_f<<<grid_for(L.n), kThreads, 0, s>>>(levd, mmov, L.n);
      } else {
        // float64 sums rounded once to float32 on store
        resize_to_level<uint8_t, double, float>(P, L, ws, mmov_u8, 1, 0, tmpd, mmov, s);
      }
    }
    // one exclusion mask for both volumes: its resize is already in levd
    if (mref_u8 && !reuse_ref && !same_mask) resize_to_level<uint8_t, double, double>(P, L, ws, mref_u8, 1, 0, tmpd, levd, s);
    const double* mref_lev = (mref_u8 && !reuse_ref) ? levd : nullptr;
    const float* mmov_lev = mmov_u8 ? mmov : nullptr;
    if (any_mask && L.nx % 4 == 0 && aligned(mref_lev, 16) && aligned(mmov_lev, 16))
      k_mask_bits_f4<<<row_grid((long long)L.nz * L.ny), kRowBlock, 0, s>>>(mref_lev, mmov_lev, bits, L.nz, L.ny,
                                                                           L.nx, reuse_ref ? 1 : 0);
    else if (any_mask)
      k_mask_bits<float><<<row_grid((long long)L.nz * L.ny), kRowBlock, 0, s>>>(
          mref_lev, nullptr, mmov_lev, nullptr, bits, L.nz, L.ny, L.nx, reuse_ref ? 1 : 0);
  }
}

static CPView cp_view(const Plan& P, const LevelPlan& L, void* ws) {
  CPView v;
  v.cp = at_off<float4>(ws, L.cp);
  v.ncx = L.ncx;
  v.ncy = L.ncy;
  v.r = P.r;
  v.w = P.w;
  return v;
}

static FieldSrc field_src(const Plan& P, int l, int mode, void* ws) {
  const LevelPlan& L = P.lv[l];
  FieldSrc f;
  memset(&f, 0, sizeof(f));
  f.mode = mode;
  f.nx = L.nx;
  f.ny = L.ny;
  f.cpv = cp_view(P, L, ws);
  f.dense = L.dense ? at_off<float4>(ws, L.dense) : nullptr;
  if (l + 1 < P.levels) {
    const LevelPlan& C = P.lv[l + 1];
    f.up.src = cp_view(P, C, ws);
    f.up.src_dense = P.dense_out[l + 1] ? at_off<float4>(ws, C.dense) : nullptr;
    f.up.src_nx = C.nx;
    f.up.src_ny = C.ny;
    f.up.wx = at_off<float>(ws, L.ux_w);
    f.up.ix = at_off<int32_t>(ws, L.ux_i);
    f.up.wy = at_off<float>(ws, L.uy_w);
    f.up.iy = at_off<int32_t>(ws, L.uy_i);
    f.up.x_first = L.up_x_first;
  }
  return f;
}

// Grid of a persistent tile kernel: as many CTAs as stay resident on the
// device at once (occupancy x SM count), at most one per tile.
// The resident-CTA count is cached per (kernel, shared memory, device);
// per_sm > 0 caps the CTAs per SM.
template <typename K>
static int persistent_grid(K kernel, size_t smem, long long ntiles, int per_sm_cap = 0) {
  struct Entry { const void* fn; size_t smem; int dev; int ctas; };
  static std::mutex mu;
  static std::vector<Entry> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  int ctas = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    for (const Entry& e : cache)
      if (e.fn == (const void*)kernel && e.smem == smem && e.dev == dev) ctas = e.ctas;
  }
  if (ctas == 0) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kAccThreads, smem);
    ctas = (sms > 0 ? sms : 1) * (per_sm > 0 ? per_sm : 1);
    std::lock_guard<std::mutex> lock(mu);
    cache.push_back(Entry{(const void*)kernel, smem, dev, ctas});
  }
  if (per_sm_cap > 0) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms > 0 && per_sm_cap * sms < ctas) ctas = per_sm_cap * sms;
  }
  return (int)(ntiles < ctas ? (ntiles > 0 ? ntiles : 1) : ctas);
}

template <int MODE, int DIFF0, bool MASK, int PREC>
static void launch_accumulate1(const IterArgs& a, long long ntiles, size_t smem, int flags, cudaStream_t s) {
  // the tile order is a template parameter: a run-time order costs the kernel registers
  auto kern = (flags & WR_LK_TILE_ORDER_X) ? k_lk_accumulate<MODE, DIFF0, MASK, PREC, 1>
                                           : k_lk_accumulate<MODE, DIFF0, MASK, PREC, 0>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int grid = persistent_grid(kern, smem, ntiles, (flags & WR_LK_CTAS_PER_SM_MASK) >> WR_LK_CTAS_PER_SM_SHIFT);
  kern<<<grid, kAccThreads, smem, s>>>(a);
}

template <int MODE, int DIFF0, int PREC>
static void launch_accumulate2(const IterArgs& a, long long ntiles, size_t smem, bool mask, int flags,
                               cudaStream_t s) {
  if (mask) launch_accumulate1<MODE, DIFF0, true, PREC>(a, ntiles, smem, flags, s);
  else launch_accumulate1<MODE, DIFF0, false, PREC>(a, ntiles, smem, flags, s);
}

// diff0: kNoDiff, or the initial-field mode of the level (CP launches only)
template <int PREC>
static void launch_accumulate(int mode, int diff0, const IterArgs& a, long long ntiles, size_t smem, bool mask,
                              int flags, cudaStream_t s) {
  switch (mode) {
    case FIELD_CP:
      switch (diff0) {
        case FIELD_UP: launch_accumulate2<FIELD_CP, FIELD_UP, PREC>(a, ntiles, smem, mask, flags, s); break;
        case FIELD_DENSE: launch_accumulate2<FIELD_CP, FIELD_DENSE, PREC>(a, ntiles, smem, mask, flags, s); break;
        case FIELD_ZERO: launch_accumulate2<FIELD_CP, FIELD_ZERO, PREC>(a, ntiles, smem, mask, flags, s); break;
        default: launch_accumulate2<FIELD_CP, kNoDiff, PREC>(a, ntiles, smem, mask, flags, s);
      }
      break;
    case FIELD_UP: launch_accumulate2<FIELD_UP, kNoDiff, PREC>(a, ntiles, smem, mask, flags, s); break;
    case FIELD_DENSE: launch_accumulate2<FIELD_DENSE, kNoDiff, PREC>(a, ntiles, smem, mask, flags, s); break;
    default: launch_accumulate2<FIELD_ZERO, kNoDiff, PREC>(a, ntiles, smem, mask, flags, s);
  }
}

// CP values of a level from its initial field
template <int MODE0>
static void cp_init(const Plan& P, const LevelPlan& L, void* ws, const FieldSrc& f, cudaStream_t s) {
  k_cp_init<MODE0><<<grid_for(L.ncp), kThreads, 0, s>>>(at_off<float4>(ws, L.cp), f, L.ncx, L.ncy, L.nz, P.r, P.w);
}

static void cp_init_dispatch(int mode, const Plan& P, const LevelPlan& L, void* ws, const FieldSrc& f,
                             cudaStream_t s) {
  switch (mode) {
    case FIELD_UP: cp_init<FIELD_UP>(P, L, ws, f, s); break;
    case FIELD_DENSE: cp_init<FIELD_DENSE>(P, L, ws, f, s); break;
    default: cp_init<FIELD_ZERO>(P, L, ws, f, s); break;
  }
}

static void build_tables(const Plan& P, void* ws, int* err_flag, cudaStream_t s) {
  for (int l = 0; l < P.levels; ++l) {
    const LevelPlan& L = P.lv[l];
    // x tables are stored tap-major ([tap][output]) for the x pass
    double* rw = at_off<double>(ws, P.tab_scratch);
    int32_t* ri = reinterpret_cast<int32_t*>(rw + (size_t)L.nx * L.tx_taps);
    k_build_table<<<(L.nx + 127) / 128, 128, 0, s>>>(rw, ri, P.nx, L.nx, RESIZE_BICUBIC, L.tx_taps);
    const long long nt = (long long)L.nx * L.tx_taps;
    k_transpose_table<<<(int)((nt + 255) / 256), 256, 0, s>>>(rw, ri, at_off<double>(ws, L.tx_w),
                                                              at_off<int32_t>(ws, L.tx_i), L.nx, L.tx_taps);
    k_build_table<<<(L.ny + 127) / 128, 128, 0, s>>>(at_off<double>(ws, L.ty_w), at_off<int32_t>(ws, L.ty_i), P.ny,
                                                      L.ny, RESIZE_BICUBIC, L.ty_taps);
    if (l + 1 < P.levels) {
      const LevelPlan& C = P.lv[l + 1];
      k_build_up_table<<<(L.nx + 127) / 128, 128, 0, s>>>(at_off<float>(ws, L.ux_w), at_off<int32_t>(ws, L.ux_i),
                                                           C.nx, L.nx, err_flag);
      k_build_up_table<<<(L.ny + 127) / 128, 128, 0, s>>>(at_off<float>(ws, L.uy_w), at_off<int32_t>(ws, L.uy_i),
                                                           C.ny, L.ny, err_flag);
    }
  }
}

// coarsest level's initial field from option["motion"] (z, y, x, 3)
static void init_field(const Plan& P, void* ws, const float* init, cudaStream_t s) {
  const LevelPlan& C = P.lv[P.levels - 1];
  float4* dense = at_off<float4>(ws, C.dense);
  float* comp = at_off<float>(ws, P.tmp_b);
  double* tmp = at_off<double>(ws, P.tmp_a);
  if (P.levels == 1) {
    // scale 1: exact copy
    for (int c = 0; c < 3; ++c)
      k_resample_x<float, double, float><<<row_grid((long long)C.nz * C.ny), kRowBlock, 0, s>>>(
          C.six, init, comp + (size_t)c * C.n, P.nz, P.ny, P.nx, C.nx, at_off<double>(ws, C.tx_w),
          at_off<int32_t>(ws, C.tx_i), C.tx_taps, 3, c);
  } else {
    for (int c = 0; c < 3; ++c)
      resize_to_level<float, double, float>(P, C, ws, init, 3, c, tmp, comp + (size_t)c * C.n, s);
  }
  double dx = (double)P.nx / (double)C.nx, dy = (double)P.ny / (double)C.ny, dz = 1.0;
  k_dense_init_pack<<<grid_for(C.n), kThreads, 0, s>>>(dense, comp, comp + C.n, comp + 2 * C.n, C.n, dx, dy, dz);
}

// Number of kernels run_register launches for a plan (kept next to the launch
// sequence it mirrors).
static int count_launches(const Plan& P, bool has_mmov, bool has_mref, bool has_init, bool reuse_ref,
                          bool same_mask) {
  int n = 0;
  const bool stored = P.precision != WR_PREC_F32;   // reduced-precision reference levels need a store pass
  for (int l = 0; l < P.levels; ++l) {
    n += 3 + (l + 1 < P.levels ? 2 : 0);                       // tables (x table built, then transposed)
    if (l == 0) n += (reuse_ref ? 1 : 2) + ((has_mmov || has_mref) ? 1 : 0);
    else n += (reuse_ref ? 3 : (stored ? 6 : 5)) + (has_mmov ? (same_mask ? 3 : 2) : 0) +
              ((has_mref && !reuse_ref && !same_mask) ? 2 : 0) + ((has_mmov || has_mref) ? 1 : 0);
  }
  if (has_init) n += (P.levels == 1 ? 3 : 6) + 1;
  for (int l = P.levels - 1; l >= 0; --l) {
    n += 1;                                                    // level begin
    if (P.dense_in[l] && !(l == P.levels - 1 && has_init)) n += 1; // dense field
    n += 1;                                                    // cp init
    n += 4 * P.iter + (P.iter >= 2 ? 1 : 0);                   // iterations + first-update check
  }
  return n + 1;                                                // final motion
}

// Pyramid, tables and initial field of one frame.
template <typename T, int PREC>
static void prepare_frame(const Plan& P, const WrLKParams* p, const T* mov, const T* ref, const uint8_t* mmov,
                          const uint8_t* mref, const float* init, void* ws, cudaStream_t s) {
  LKState* st = at_off<LKState>(ws, P.state);
  int* err_flag = reinterpret_cast<int*>(reinterpret_cast<char*>(st) + sizeof(LKState));
  cudaMemsetAsync(err_flag, 0, sizeof(int), s);
  build_tables(P, ws, err_flag, s);
  build_pyramid<T, PREC>(P, ws, mov, ref, mmov, mref, (p->flags & WR_LK_REUSE_REFERENCE) != 0, s);
  if (init) init_field(P, ws, init, s);
}

// Multiplier of div_magic for divisor d and dividends below nmax: ceil(2^32 / d)
// when every such dividend n has n * d <= 2^32, else 0 (plain division).
static uint32_t host_div_magic(long long d, long long nmax) {
  if (d <= 1 || (nmax - 1) * d > (1LL << 32)) return 0;
  return (uint32_t)(((1ULL << 32) + (unsigned long long)d - 1) / (unsigned long long)d);
}

// Start of level l for one frame: control state, initial field, CP values and
// the fused kernel's arguments (field = the level's initial field; mode0 is
// returned in *mode0).
static IterArgs begin_level(const Plan& P, int l, void* ws, bool has_init, bool mask, bool has_mmov, int* mode0,
                            cudaStream_t s) {
  const LevelPlan& L = P.lv[l];
  LKState* st = at_off<LKState>(ws, P.state);
  const bool coarsest = l == P.levels - 1;
  k_level_begin<<<1, 1, 0, s>>>(st, l, coarsest ? 1 : 0);
  int m0 = coarsest ? (has_init ? FIELD_DENSE : FIELD_ZERO) : FIELD_UP;
  if (P.dense_in[l] && !(coarsest && has_init)) {
    // a level without update keeps its dense initial field (and the next
    // finer level starts from that field, materialised)
    FieldSrc f = field_src(P, l, m0, ws);
    float4* dense = at_off<float4>(ws, L.dense);
    const int g = row_grid((long long)L.nz * L.ny);
    if (m0 == FIELD_UP) k_dense_from<FIELD_UP><<<g, kRowBlock, 0, s>>>(dense, f, L.nx, L.ny, L.nz);
    else if (m0 == FIELD_ZERO) k_dense_from<FIELD_ZERO><<<g, kRowBlock, 0, s>>>(dense, f, L.nx, L.ny, L.nz);
    m0 = FIELD_DENSE;
  }
  const FieldSrc f0 = field_src(P, l, m0, ws);
  cp_init_dispatch(m0, P, L, ws, f0, s);
  IterArgs a;
  memset(&a, 0, sizeof(a));
  a.st = st;
  a.ref = at_off<void>(ws, L.ref);
  a.mov.g = at_off<void>(ws, L.movg);
  a.mov.nx = L.nx;
  a.mov.ny = L.ny;
  a.mov.nz = L.nz;
  a.mbits = mask ? at_off<uint8_t>(ws, L.mbits) : nullptr;
  a.mmov = has_mmov ? at_off<float>(ws, L.mmov) : nullptr;
  a.sums = at_off<float>(ws, L.sums);
  a.errpart = at_off<double>(ws, L.errpart);
  a.penpart = at_off<double>(ws, L.penpart);
  a.cpv = cp_view(P, L, ws);
  a.r = P.r;
  a.w = P.w;
  a.ntx = L.ntx;
  a.nty = L.nty;
  a.zratio = L.zratio;
  a.nz_magic = host_div_magic(L.nz, L.nblk);
  a.ntx_magic = host_div_magic(L.ntx, (long long)L.ntx * L.nty);
  // level constants of the sampling loop (tap clamps, plane strides, face tests)
  a.nxm1 = L.nx - 1;
  a.nym1 = L.ny - 1;
  a.nxm2 = L.nx - 2;
  a.nym2 = L.ny - 2;
  a.bzmax = L.nz > 2 ? L.nz - 2 : 0;
  a.plane = (uint32_t)L.nx * (uint32_t)L.ny;
  a.oz1 = L.nz > 1 ? a.plane : 0u;   // a single slice reads its only plane twice
  a.fnx = (float)L.nx;
  a.fny = (float)L.ny;
  a.fnz = (float)L.nz;
  a.fnxm1 = (float)(L.nx - 1);
  a.fnym1 = (float)(L.ny - 1);
  a.fnzm1 = (float)(L.nz - 1);
  a.fzmax = L.nz > 1 ? 1.f : 0.f;
  a.field = f0;
  a.field0 = f0;
  *mode0 = m0;
  return a;
}

// Full-resolution motion (and the warped frame), stats.
template <typename T>
static void finish_frame(const Plan& P, void* ws, const T* mov, float* out, float* warped, WrLKStats* stats,
                         cudaStream_t s) {
  const LevelPlan& L0 = P.lv[0];
  const int g0 = row_grid((long long)L0.nz * L0.ny);
  const int mode_out = P.dense_out[0] ? FIELD_DENSE : FIELD_CP;
  const FieldSrc f = field_src(P, 0, mode_out, ws);
  if (warped) {
    // the full-resolution motion and mov warped by it, in one pass
    if (mode_out == FIELD_DENSE)
      k_write_motion_warp<FIELD_DENSE, T><<<g0, kRowBlock, 0, s>>>(out, warped, mov, f, L0.nx, L0.ny, L0.nz);
    else
      k_write_motion_warp<FIELD_CP, T><<<g0, kRowBlock, 0, s>>>(out, warped, mov, f, L0.nx, L0.ny, L0.nz);
  } else if (mode_out == FIELD_DENSE) {
    k_write_motion<FIELD_DENSE><<<g0, kRowBlock, 0, s>>>(out, f, L0.nx, L0.ny, L0.nz);
  } else {
    k_write_motion<FIELD_CP><<<g0, kRowBlock, 0, s>>>(out, f, L0.nx, L0.ny, L0.nz);
  }
  LKState* st = at_off<LKState>(ws, P.state);
  if (stats) cudaMemcpyAsync(stats, &st->stats, sizeof(WrLKStats), cudaMemcpyDeviceToDevice, s);
}

// error_log snapshot of one iteration slot (motion and warped moving level)
template <int PREC>
static void snapshot(int mode, const LKState* st, const FieldSrc& f, const void* movg, const LevelPlan& L,
                     float* motion, float* warped, cudaStream_t s) {
  const typename Store<PREC>::V4* g = static_cast<const typename Store<PREC>::V4*>(movg);
  const int grid = row_grid((long long)L.nz * L.ny);
  switch (mode) {
    case FIELD_CP: k_snapshot<FIELD_CP, PREC><<<grid, kRowBlock, 0, s>>>(st, f, g, L.nx, L.ny, L.nz, motion, warped); break;
    case FIELD_UP: k_snapshot<FIELD_UP, PREC><<<grid, kRowBlock, 0, s>>>(st, f, g, L.nx, L.ny, L.nz, motion, warped); break;
    case FIELD_DENSE:
      k_snapshot<FIELD_DENSE, PREC><<<grid, kRowBlock, 0, s>>>(st, f, g, L.nx, L.ny, L.nz, motion, warped);
      break;
    default: k_snapshot<FIELD_ZERO, PREC><<<grid, kRowBlock, 0, s>>>(st, f, g, L.nx, L.ny, L.nz, motion, warped);
  }
}

template <typename T, int PREC>
static int run_register(const Plan& P, const WrLKParams* p, const T* mov, const T* ref, const uint8_t* mmov,
                        const uint8_t* mref, const float* init, float* out, float* warped, WrLKStats* stats, void* ws,
                        cudaStream_t s, WrProfile* prof, const WrSnapshots* snap = nullptr) {
  int recorded = 0;
  LKState* st = at_off<LKState>(ws, P.state);
  prepare_frame<T, PREC>(P, p, mov, ref, mmov, mref, init, ws, s);
  const bool reuse_ref = (p->flags & WR_LK_REUSE_REFERENCE) != 0;
  const bool mask = mmov || mref;
  const double sps = p->smoothPenalty * (double)((2 * P.r + 1) * (2 * P.r + 1));
  const float sps_f = (float)sps;
  for (int l = P.levels - 1; l >= 0; --l) {
    const LevelPlan& L = P.lv[l];
    int mode0;
    IterArgs a = begin_level(P, l, ws, init != nullptr, mask, mmov != nullptr, &mode0, s);
    const FieldSrc f0 = a.field0;
    const int forced = p->forced_updates[l];
    if (snap && (snap->level_ref[l] || snap->level_mov[l]))
      k_level_images<PREC><<<grid_for(L.n), kThreads, 0, s>>>(static_cast<const typename Store<PREC>::V1*>(a.ref),
                                                              static_cast<const typename Store<PREC>::V4*>(a.mov.g),
                                                              L.n, snap->level_ref[l], snap->level_mov[l]);
    for (int it = 0; it < P.iter; ++it) {
      const int mode = it == 0 ? mode0 : FIELD_CP;
      // the launch after the level's first update also measures max |new - initial|
      const int diff0 = it == 1 ? mode0 : kNoDiff;
      a.field = it == 0 ? f0 : field_src(P, l, FIELD_CP, ws);
      if (snap && snap->save_ite > 0 && it % snap->save_ite == 0 && it / snap->save_ite < snap->capacity) {
        const size_t slot = (size_t)(it / snap->save_ite) * L.n;
        snapshot<PREC>(mode, st, a.field, a.mov.g, L, snap->motion[l] ? snap->motion[l] + 3 * slot : nullptr,
                       snap->warped[l] ? snap->warped[l] + slot : nullptr, s);
      }
      const size_t smem = accumulate_smem(P.w, diff0 == FIELD_UP);
      const bool rec = prof && recorded < prof->capacity;
      if (rec) cudaEventRecord((cudaEvent_t)prof->acc_begin[recorded], s);
      launch_accumulate<PREC>(mode, diff0, a, L.nblk, smem, mask, p->flags, s);
      if (rec) cudaEventRecord((cudaEvent_t)prof->acc_end[recorded++], s);
      if (diff0 != kNoDiff) k_first_post<<<1, 1, 0, s>>>(st, l, forced, kMotionTol);
      k_decide<<<1, 1024, 0, s>>>(st, a.errpart, a.penpart, L.nblk, (double)L.n, sps, l, it, P.iter, p->tol, forced);
      if (PREC == WR_PREC_F32)
        k_update<false><<<grid_for(L.ncp), kThreads, 0, s>>>(st, at_off<float4>(ws, L.cp), a.sums, L.ncp, sps, sps_f,
                                                              (double)p->movRange, L.zratio_d);
      else
        k_update<true><<<grid_for(L.ncp), kThreads, 0, s>>>(st, at_off<float4>(ws, L.cp), a.sums, L.ncp, sps, sps_f,
                                                             (double)p->movRange, L.zratio_d);
      k_post<<<1, 1, 0, s>>>(st, l, forced, it == 0 ? 1 : 0, kMotionTol);
    }
  }
  finish_frame<T>(P, ws, mov, out, warped, stats, s);
  if (prof) {
    prof->recorded = recorded;
    prof->launches = count_launches(P, mmov != nullptr, mref != nullptr, init != nullptr, reuse_ref,
                                    mmov != nullptr && mmov == mref && !reuse_ref);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "wr_lk_register launch");
  return WR_OK;
}

// ---------------------------------------------------------------------------
// batched registration
// ---------------------------------------------------------------------------

template <int MODE, int DIFF0, bool MASK, int PREC>
static void launch_batch1(const BatchIter& b, long long ntiles, size_t smem, int flags, cudaStream_t s) {
  auto kern = k_lk_accumulate_batch<MODE, DIFF0, MASK, PREC>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int grid = persistent_grid(kern, smem, ntiles, (flags & WR_LK_CTAS_PER_SM_MASK) >> WR_LK_CTAS_PER_SM_SHIFT);
  kern<<<grid, kAccThreads, smem, s>>>(b);
}

template <int MODE, int DIFF0, int PREC>
static void launch_batch2(const BatchIter& b, long long ntiles, size_t smem, bool mask, int flags, cudaStream_t s) {
  if (mask) launch_batch1<MODE, DIFF0, true, PREC>(b, ntiles, smem, flags, s);
  else launch_batch1<MODE, DIFF0, false, PREC>(b, ntiles, smem, flags, s);
}

template <int PREC>
static void launch_batch(int mode, int diff0, const BatchIter& b, long long ntiles, size_t smem, bool mask, int flags,
                         cudaStream_t s) {
  switch (mode) {
    case FIELD_CP:
      switch (diff0) {
        case FIELD_UP: launch_batch2<FIELD_CP, FIELD_UP, PREC>(b, ntiles, smem, mask, flags, s); break;
        case FIELD_DENSE: launch_batch2<FIELD_CP, FIELD_DENSE, PREC>(b, ntiles, smem, mask, flags, s); break;
        case FIELD_ZERO: launch_batch2<FIELD_CP, FIELD_ZERO, PREC>(b, ntiles, smem, mask, flags, s); break;
        default: launch_batch2<FIELD_CP, kNoDiff, PREC>(b, ntiles, smem, mask, flags, s);
      }
      break;
    case FIELD_UP: launch_batch2<FIELD_UP, kNoDiff, PREC>(b, ntiles, smem, mask, flags, s); break;
    case FIELD_DENSE: launch_batch2<FIELD_DENSE, kNoDiff, PREC>(b, ntiles, smem, mask, flags, s); break;
    default: launch_batch2<FIELD_ZERO, kNoDiff, PREC>(b, ntiles, smem, mask, flags, s);
  }
}

// Tiles from which a frame-level of a batch takes its own launch of the
// single-volume iteration kernel: four rounds of a full-GPU persistent grid
// (1184 and 4736 measured the same on the uneven batch, 4736 2 % slower on 16
// frames of 64x256x256).  Smaller frame-levels share one launch
// (k_lk_accumulate_batch), which fills the GPU with several frames but reads
// each frame's parameters by a runtime index (11 % more instructions per
// voxel, measured on an uneven batch).
constexpr long long kOwnLaunchTiles = 4LL * 148 * 4;

// Frames may differ in shape, patch radius, number of levels, iterations and
// every other solver parameter except the precision and the launch-shape
// flags.  Level l (0 = finest) of every frame that has it runs together; an
// iteration launch holds the frames with that many iterations left, grouped
// by the kernel variant their field needs (a frame's first level starts from
// its initial field while frames with more levels up-sample theirs).
template <typename T, int PREC>
static int run_batch(const Plan* plans, const size_t* offs, const WrLKItem* items, int n, const WrLKParams* params,
                     void* workspace, cudaStream_t s) {
  void* ws[kMaxBatch];
  int max_levels = 0, max_iter = 0;
  for (int i = 0; i < n; ++i) {
    ws[i] = static_cast<char*>(workspace) + offs[i];
    prepare_frame<T, PREC>(plans[i], &params[i], (const T*)items[i].mov.data, (const T*)items[i].ref.data,
                           items[i].excl_mask_mov, items[i].excl_mask_ref, items[i].motion_init, ws[i], s);
    max_levels = std::max(max_levels, plans[i].levels);
    max_iter = std::max(max_iter, plans[i].iter);
  }
  const bool has_init = items[0].motion_init != nullptr;
  const bool has_mmov = items[0].excl_mask_mov != nullptr;
  const bool mask = has_mmov || items[0].excl_mask_ref != nullptr;
  const int flags = params[0].flags;
  const int order = (flags & WR_LK_TILE_ORDER_X) ? 1 : 0;
  static thread_local BatchIter b;
  BatchDecide bd;
  BatchUpdate bu;
  BatchState bs;
  for (int l = max_levels - 1; l >= 0; --l) {
    IterArgs args[kMaxBatch];
    FieldSrc f0[kMaxBatch];
    int mode0[kMaxBatch];
    for (int i = 0; i < n; ++i)
      if (l < plans[i].levels) {
        args[i] = begin_level(plans[i], l, ws[i], has_init, mask, has_mmov, &mode0[i], s);
        f0[i] = args[i].field0;
      }
    for (int it = 0; it < max_iter; ++it) {
      int act[kMaxBatch], na = 0;
      for (int i = 0; i < n; ++i)
        if (l < plans[i].levels && it < plans[i].iter) act[na++] = i;
      if (na == 0) break;
      // the fused iteration, one launch per (field mode, first-difference mode) group
      bool done[kMaxBatch] = {};
      for (int g = 0; g < na; ++g) {
        if (done[g]) continue;
        const int i0 = act[g];
        const int mode = it == 0 ? mode0[i0] : FIELD_CP;
        const int diff0 = it == 1 ? mode0[i0] : kNoDiff;
        memset(&b, 0, sizeof(b));
        b.order = order;
        size_t smem = 0;
        int m = 0;
        b.tile_start[0] = 0;
        for (int h = g; h < na; ++h) {
          const int i = act[h];
          if (done[h] || (it == 0 ? mode0[i] : FIELD_CP) != mode || (it == 1 ? mode0[i] : kNoDiff) != diff0) continue;
          done[h] = true;
          IterArgs ai = args[i];
          ai.field = it == 0 ? f0[i] : field_src(plans[i], l, FIELD_CP, ws[i]);
          const long long nblk = plans[i].lv[l].nblk;
          if (nblk >= kOwnLaunchTiles) {
            // enough tiles to fill the GPU alone: the single-volume kernel,
            // whose frame parameters are constant operands (same results)
            launch_accumulate<PREC>(mode, diff0, ai, nblk, accumulate_smem(plans[i].w, diff0 == FIELD_UP), mask,
                                    flags, s);
            continue;
          }
          b.item[m] = ai;
          b.tile_start[m + 1] = b.tile_start[m] + (int)nblk;
          smem = std::max(smem, accumulate_smem(plans[i].w, diff0 == FIELD_UP));
          ++m;
        }
        b.n = m;
        if (m > 0) launch_batch<PREC>(mode, diff0, b, b.tile_start[m], smem, mask, flags, s);
      }
      memset(&bd, 0, sizeof(bd));
      memset(&bu, 0, sizeof(bu));
      memset(&bs, 0, sizeof(bs));
      bd.n = bu.n = bs.n = na;
      long long max_ncp = 1;
      for (int k = 0; k < na; ++k) {
        const int i = act[k];
        const Plan& P = plans[i];
        const LevelPlan& L = P.lv[l];
        const double sps = params[i].smoothPenalty * (double)((2 * P.r + 1) * (2 * P.r + 1));
        bd.st[k] = bu.st[k] = bs.st[k] = args[i].st;
        bd.errpart[k] = args[i].errpart;
        bd.penpart[k] = args[i].penpart;
        bd.nblk[k] = L.nblk;
        bd.n_vox[k] = (double)L.n;
        bd.sps[k] = sps;
        bd.tol[k] = params[i].tol;
        bd.iter[k] = P.iter;
        bd.forced[k] = bs.forced[k] = params[i].forced_updates[l];
        bu.cp[k] = at_off<float4>(ws[i], L.cp);
        bu.sums[k] = args[i].sums;
        bu.ncp[k] = L.ncp;
        bu.sps[k] = sps;
        bu.sps_f[k] = (float)sps;
        bu.mov_range[k] = (double)params[i].movRange;
        bu.zratio_d[k] = L.zratio_d;
        max_ncp = std::max(max_ncp, L.ncp);
      }
      const dim3 ugrid((unsigned)((max_ncp + kThreads - 1) / kThreads), (unsigned)na);
      if (it == 1) k_first_post_batch<<<1, kMaxBatch, 0, s>>>(bs, l);
      k_decide_batch<<<na, 1024, 0, s>>>(bd, l, it);
      if (PREC == WR_PREC_F32) k_update_batch<false><<<ugrid, kThreads, 0, s>>>(bu);
      else k_update_batch<true><<<ugrid, kThreads, 0, s>>>(bu);
      k_post_batch<<<1, kMaxBatch, 0, s>>>(bs, l, it == 0 ? 1 : 0);
    }
  }
  for (int i = 0; i < n; ++i)
    finish_frame<T>(plans[i], ws[i], (const T*)items[i].mov.data, items[i].motion_out, items[i].warped_out,
                    items[i].stats, s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "wr_lk_register_batch launch");
  return WR_OK;
}

// ---------------------------------------------------------------------------
// penalty factor without allocation: per-block partial sums in a static array
// ---------------------------------------------------------------------------

// Each block of the no-alloc variant reduces a fixed 16,384-voxel span, so a
// volume needs ceil(n / 16384) partial slots; 8,192 slots of 4 doubles
// (256 KiB, resident on every device that loads the library) cover volumes of
// up to 134,217,728 voxels (128 x 1024 x 1024).
constexpr int kNoAllocVoxelsPerBlock = kThreads * 64;
constexpr int kNoAllocSlots = 8192;
constexpr long long kNoAllocMaxVoxels = (long long)kNoAllocSlots * kNoAllocVoxelsPerBlock;
static __device__ __align__(256) double g_noalloc_partials[kNoAllocSlots * 4];

static std::mutex g_noalloc_mu;
static double* g_noalloc_dev_ptr[128] = {};

// Device address of the static scratch for the current device, looked up once
// per device (host code may not use the symbol itself as a device pointer).
static int noalloc_partials(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "wr_penalty_factor_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= 128) return fail(WR_E_PARAM, "wr_penalty_factor_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_dev_ptr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) return cuda_fail(e, "wr_penalty_factor_noalloc: cudaGetSymbolAddress");
    g_noalloc_dev_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_dev_ptr[dev];
  return WR_OK;
}

template <int PREC>
static int dispatch_dtype(const Plan& P, const WrLKParams* p, const WrVolume* mov, const WrVolume* ref,
                          const uint8_t* mmov, const uint8_t* mref, const float* init, float* out, float* warped,
                          WrLKStats* stats, void* ws, cudaStream_t s, WrProfile* prof, const WrSnapshots* snap) {
  switch (mov->dtype) {
    case WR_U16:
      return run_register<uint16_t, PREC>(P, p, (const uint16_t*)mov->data, (const uint16_t*)ref->data, mmov, mref,
                                          init, out, warped, stats, ws, s, prof, snap);
    case WR_U8:
      return run_register<uint8_t, PREC>(P, p, (const uint8_t*)mov->data, (const uint8_t*)ref->data, mmov, mref, init,
                                         out, warped, stats, ws, s, prof, snap);
    default:
      return run_register<float, PREC>(P, p, (const float*)mov->data, (const float*)ref->data, mmov, mref, init, out,
                                       warped, stats, ws, s, prof, snap);
  }
}

static int check_volume(const WrVolume* v, const char* name) {
  if (!v || !v->data) return fail(WR_E_NULL, (std::string(name) + " is NULL").c_str());
  if (v->dtype != WR_U8 && v->dtype != WR_U16 && v->dtype != WR_F32)
    return fail(WR_E_DTYPE, (std::string(name) + ": dtype must be WR_U8, WR_U16 or WR_F32").c_str());
  if (v->nz < 1 || v->ny < 1 || v->nx < 1) return fail(WR_E_SHAPE, (std::string(name) + ": empty volume").c_str());
  return WR_OK;
}

}  // namespace wr

using namespace wr;

#include "wr_xres_host.inc"

extern "C" {

int wr_abi_version(void) { return WR_ABI_VERSION; }

const char* wr_last_error(void) { return g_last_error.c_str(); }

int wr_lk_workspace_size(int32_t nz, int32_t ny, int32_t nx, const WrLKParams* p, size_t* bytes) {
  if (!p || !bytes) return fail(WR_E_NULL, "params or bytes is NULL");
  Plan P;
  const char* why;
  int rc = make_plan(nz, ny, nx, p, true, true, true, &P, &why);
  if (rc) return fail(rc, why);
  *bytes = P.total;
  return WR_OK;
}

// Plans and workspace offsets of a batch (validates the items; with
// sizes_only the data and output pointers are not looked at).
static int batch_plans(const WrLKItem* items, int32_t n, const WrLKParams* params, Plan* plans, size_t* offs,
                       size_t* total, bool sizes_only) {
  if (!items || !params) return fail(WR_E_NULL, "items or params is NULL");
  if (n < 1 || n > WR_MAX_BATCH) return fail(WR_E_PARAM, "batch size must be 1..WR_MAX_BATCH");
  size_t cur = 0;
  const int launch_bits = WR_LK_TILE_ORDER_X | WR_LK_CTAS_PER_SM_MASK;
  for (int i = 0; i < n; ++i) {
    const WrLKItem& it = items[i];
    int rc;
    if (sizes_only) {
      WrVolume m = it.mov, r = it.ref;
      m.data = r.data = items;   // any non-null address: only shapes and dtypes are checked
      if ((rc = check_volume(&m, "mov"))) return rc;
      if ((rc = check_volume(&r, "ref"))) return rc;
    } else {
      if ((rc = check_volume(&it.mov, "mov"))) return rc;
      if ((rc = check_volume(&it.ref, "ref"))) return rc;
      if (!it.motion_out) return fail(WR_E_NULL, "motion_out is NULL");
    }
    if (it.mov.nz != it.ref.nz || it.mov.ny != it.ref.ny || it.mov.nx != it.ref.nx)
      return fail(WR_E_SHAPE, "mov and ref shapes differ");
    if (it.mov.dtype != it.ref.dtype || it.mov.dtype != items[0].mov.dtype)
      return fail(WR_E_DTYPE, "every volume of a batch must have one dtype");
    if ((it.excl_mask_mov != nullptr) != (items[0].excl_mask_mov != nullptr) ||
        (it.excl_mask_ref != nullptr) != (items[0].excl_mask_ref != nullptr) ||
        (it.motion_init != nullptr) != (items[0].motion_init != nullptr))
      return fail(WR_E_PARAM, "the frames of a batch must agree on which masks and initial fields are given");
    if (params[i].precision != params[0].precision || (params[i].flags & launch_bits) != (params[0].flags & launch_bits))
      return fail(WR_E_PARAM, "the frames of a batch must agree on the precision and the launch-shape flags");
    const char* why;
    rc = make_plan(it.mov.nz, it.mov.ny, it.mov.nx, &params[i], true, true, true, &plans[i], &why);
    if (rc) return fail(rc, why);
    offs[i] = cur;
    cur = align_up(cur + plans[i].total);
  }
  *total = cur;
  return WR_OK;
}

int wr_lk_batch_each_workspace_size(const WrLKItem* items, const WrLKParams* params, int32_t n, size_t* bytes) {
  if (!bytes) return fail(WR_E_NULL, "bytes is NULL");
  static thread_local Plan plans[WR_MAX_BATCH];
  size_t offs[WR_MAX_BATCH];
  return batch_plans(items, n, params, plans, offs, bytes, true);
}

int wr_lk_register_batch_each(const WrLKItem* items, const WrLKParams* params, int32_t n, void* workspace,
                              size_t workspace_bytes, void* stream) {
  static thread_local Plan plans[WR_MAX_BATCH];
  size_t offs[WR_MAX_BATCH], total = 0;
  int rc = batch_plans(items, n, params, plans, offs, &total, false);
  if (rc) return rc;
  if (!workspace) return fail(WR_E_NULL, "workspace is NULL");
  if (reinterpret_cast<uintptr_t>(workspace) % 256) return fail(WR_E_WORKSPACE, "workspace must be 256-byte aligned");
  if (workspace_bytes < total) return fail(WR_E_WORKSPACE, "workspace smaller than wr_lk_batch_workspace_size");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int dtype = items[0].mov.dtype;
#define WR_BATCH_DISPATCH(PRECV)                                                                        \
  switch (dtype) {                                                                                      \
    case WR_U16: return run_batch<uint16_t, PRECV>(plans, offs, items, n, params, workspace, s);        \
    case WR_U8: return run_batch<uint8_t, PRECV>(plans, offs, items, n, params, workspace, s);          \
    default: return run_batch<float, PRECV>(plans, offs, items, n, params, workspace, s);                \
  }
  switch (params[0].precision) {
    case WR_PREC_F16: WR_BATCH_DISPATCH(WR_PREC_F16)
    case WR_PREC_BF16: WR_BATCH_DISPATCH(WR_PREC_BF16)
    default: WR_BATCH_DISPATCH(WR_PREC_F32)
  }
#undef WR_BATCH_DISPATCH
}

// one parameter set for every frame: the per-frame form with n copies
static int replicate_params(const WrLKParams* p, int32_t n, WrLKParams* out) {
  if (!p) return fail(WR_E_NULL, "params is NULL");
  if (n < 1 || n > WR_MAX_BATCH) return fail(WR_E_PARAM, "batch size must be 1..WR_MAX_BATCH");
  for (int i = 0; i < n; ++i) out[i] = *p;
  return WR_OK;
}

int wr_lk_batch_workspace_size(const WrLKItem* items, int32_t n, const WrLKParams* p, size_t* bytes) {
  WrLKParams ps[WR_MAX_BATCH];
  int rc = replicate_params(p, n, ps);
  return rc ? rc : wr_lk_batch_each_workspace_size(items, ps, n, bytes);
}

int wr_lk_register_batch(const WrLKItem* items, int32_t n, const WrLKParams* p, void* workspace,
                         size_t workspace_bytes, void* stream) {
  WrLKParams ps[WR_MAX_BATCH];
  int rc = replicate_params(p, n, ps);
  return rc ? rc : wr_lk_register_batch_each(items, ps, n, workspace, workspace_bytes, stream);
}

int wr_lk_register(const WrVolume* mov, const WrVolume* ref, const uint8_t* excl_mask_mov,
                   const uint8_t* excl_mask_ref, const WrLKParams* p, const float* motion_init, float* motion_out,
                   WrLKStats* stats, void* workspace, size_t workspace_bytes, void* stream) {
  return wr_lk_register_profiled(mov, ref, excl_mask_mov, excl_mask_ref, p, motion_init, motion_out, stats,
                                 workspace, workspace_bytes, stream, nullptr);
}

// getMotion, optionally followed by correctMotion of mov (warped != null),
// with optional per-launch events around the fused iteration kernel.
static int register_common(const WrVolume* mov, const WrVolume* ref, const uint8_t* excl_mask_mov,
                           const uint8_t* excl_mask_ref, const WrLKParams* p, const float* motion_init,
                           float* motion_out, float* warped_out, WrLKStats* stats, void* workspace,
                           size_t workspace_bytes, void* stream, WrProfile* prof, const WrSnapshots* snap = nullptr) {
  int rc;
  if ((rc = check_volume(mov, "mov"))) return rc;
  if ((rc = check_volume(ref, "ref"))) return rc;
  if (!p) return fail(WR_E_NULL, "params is NULL");
  if (!motion_out) return fail(WR_E_NULL, "motion_out is NULL");
  if (!workspace) return fail(WR_E_NULL, "workspace is NULL");
  if (mov->nz != ref->nz || mov->ny != ref->ny || mov->nx != ref->nx)
    return fail(WR_E_SHAPE, "mov and ref shapes differ");
  if (mov->dtype != ref->dtype) return fail(WR_E_DTYPE, "mov and ref dtypes differ");
  if (reinterpret_cast<uintptr_t>(workspace) % 256) return fail(WR_E_WORKSPACE, "workspace must be 256-byte aligned");
  Plan P;
  const char* why;
  rc = make_plan(mov->nz, mov->ny, mov->nx, p, true, true, true, &P, &why);
  if (rc) return fail(rc, why);
  if (workspace_bytes < P.total) return fail(WR_E_WORKSPACE, "workspace smaller than wr_lk_workspace_size");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (p->precision) {
    case WR_PREC_F16:
      return dispatch_dtype<WR_PREC_F16>(P, p, mov, ref, excl_mask_mov, excl_mask_ref, motion_init, motion_out,
                                         warped_out, stats, workspace, s, prof, snap);
    case WR_PREC_BF16:
      return dispatch_dtype<WR_PREC_BF16>(P, p, mov, ref, excl_mask_mov, excl_mask_ref, motion_init, motion_out,
                                          warped_out, stats, workspace, s, prof, snap);
    default:
      return dispatch_dtype<WR_PREC_F32>(P, p, mov, ref, excl_mask_mov, excl_mask_ref, motion_init, motion_out,
                                         warped_out, stats, workspace, s, prof, snap);
  }
}

int wr_lk_register_profiled(const WrVolume* mov, const WrVolume* ref, const uint8_t* excl_mask_mov,
                            const uint8_t* excl_mask_ref, const WrLKParams* p, const float* motion_init,
                            float* motion_out, WrLKStats* stats, void* workspace, size_t workspace_bytes,
                            void* stream, WrProfile* prof) {
  return register_common(mov, ref, excl_mask_mov, excl_mask_ref, p, motion_init, motion_out, nullptr, stats,
                         workspace, workspace_bytes, stream, prof);
}

int wr_lk_register_snapshots(const WrVolume* mov, const WrVolume* ref, const uint8_t* excl_mask_mov,
                             const uint8_t* excl_mask_ref, const WrLKParams* p, const float* motion_init,
                             float* motion_out, WrLKStats* stats, void* workspace, size_t workspace_bytes,
                             void* stream, const WrSnapshots* snap) {
  if (snap && (snap->save_ite < 1 || snap->capacity < 0)) return fail(WR_E_PARAM, "snapshots: save_ite >= 1, capacity >= 0");
  return register_common(mov, ref, excl_mask_mov, excl_mask_ref, p, motion_init, motion_out, nullptr, stats,
                         workspace, workspace_bytes, stream, nullptr, snap);
}

int wr_lk_register_warp(const WrVolume* mov, const WrVolume* ref, const uint8_t* excl_mask_mov,
                        const uint8_t* excl_mask_ref, const WrLKParams* p, const float* motion_init, float* motion_out,
                        float* warped_out, WrLKStats* stats, void* workspace, size_t workspace_bytes, void* stream,
                        WrProfile* prof) {
  if (!warped_out) return fail(WR_E_NULL, "warped_out is NULL");
  return register_common(mov, ref, excl_mask_mov, excl_mask_ref, p, motion_init, motion_out, warped_out, stats,
                         workspace, workspace_bytes, stream, prof);
}

int wr_warp_trilinear(const WrVolume* src, const float* motion, float* out, void* stream) {
  int rc;
  if ((rc = check_volume(src, "src"))) return rc;
  if (!motion || !out) return fail(WR_E_NULL, "motion or out is NULL");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long rows = (long long)src->nz * src->ny;
  if (rows >= (1LL << 31)) return fail(WR_E_SHAPE, "src has 2^31 rows or more");
  const int g = row_grid(rows);
  switch (src->dtype) {
    case WR_U16:
      k_warp<uint16_t><<<g, kRowBlock, 0, s>>>((const uint16_t*)src->data, motion, out, src->nz, src->ny, src->nx);
      break;
    case WR_U8:
      k_warp<uint8_t><<<g, kRowBlock, 0, s>>>((const uint8_t*)src->data, motion, out, src->nz, src->ny, src->nx);
      break;
    default:
      k_warp<float><<<g, kRowBlock, 0, s>>>((const float*)src->data, motion, out, src->nz, src->ny, src->nx);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "wr_warp_trilinear launch");
  return WR_OK;
}

int wr_penalty_factor_scratch(int32_t nz, int32_t ny, int32_t nx, size_t* bytes) {
  if (!bytes) return fail(WR_E_NULL, "bytes is NULL");
  if (nz < 1 || ny < 1 || nx < 1) return fail(WR_E_SHAPE, "empty volume");
  *bytes = (size_t)grid_for((long long)nz * ny * nx) * 4 * sizeof(double);
  return WR_OK;
}

int wr_penalty_factor(const WrVolume* ref, const uint8_t* excl_mask_ref, double* factor_out, void* scratch,
                      size_t scratch_bytes, void* stream) {
  int rc;
  if ((rc = check_volume(ref, "ref"))) return rc;
  if (!factor_out || !scratch) return fail(WR_E_NULL, "factor_out or scratch is NULL");
  if (ref->nx < 3 || ref->ny < 3) return fail(WR_E_SHAPE, "ref needs at least 3 voxels along x and y");
  long long n = (long long)ref->nz * ref->ny * ref->nx;
  int nblk = grid_for(n);
  if (scratch_bytes < (size_t)nblk * 4 * sizeof(double)) return fail(WR_E_WORKSPACE, "scratch too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* part = static_cast<double*>(scratch);
  switch (ref->dtype) {
    case WR_U16:
      k_penalty_partial<uint16_t><<<nblk, kThreads, 0, s>>>((const uint16_t*)ref->data, excl_mask_ref, part, ref->nz, ref->ny, ref->nx);
      break;
    case WR_U8:
      k_penalty_partial<uint8_t><<<nblk, kThreads, 0, s>>>((const uint8_t*)ref->data, excl_mask_ref, part, ref->nz, ref->ny, ref->nx);
      break;
    default:
      k_penalty_partial<float><<<nblk, kThreads, 0, s>>>((const float*)ref->data, excl_mask_ref, part, ref->nz, ref->ny, ref->nx);
  }
  k_penalty_final<<<1, 1024, 0, s>>>(part, nblk, factor_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "wr_penalty_factor launch");
  return WR_OK;
}

int wr_penalty_factor_noalloc(const WrVolume* ref, const uint8_t* excl_mask_ref, double* factor_out,
                              void* stream) {
  int rc;
  if ((rc = check_volume(ref, "ref"))) return rc;
  if (!factor_out) return fail(WR_E_NULL, "factor_out is NULL");
  if (ref->nx < 3 || ref->ny < 3) return fail(WR_E_SHAPE, "ref needs at least 3 voxels along x and y");
  const long long n = (long long)ref->nz * ref->ny * ref->nx;
  if (n > kNoAllocMaxVoxels)
    return fail(WR_E_SHAPE, "wr_penalty_factor_noalloc: volume exceeds the 134217728-voxel capacity of its static "
                            "scratch; use wr_penalty_factor with caller-provided scratch");
  double* part = nullptr;
  if ((rc = noalloc_partials(&part))) return rc;
  const int nblk = (int)((n + kNoAllocVoxelsPerBlock - 1) / kNoAllocVoxelsPerBlock);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // every slot read by the final reduction is written by this call's blocks
  switch (ref->dtype) {
    case WR_U16:
      k_penalty_partial<uint16_t><<<nblk, kThreads, 0, s>>>((const uint16_t*)ref->data, excl_mask_ref, part, ref->nz, ref->ny, ref->nx);
      break;
    case WR_U8:
      k_penalty_partial<uint8_t><<<nblk, kThreads, 0, s>>>((const uint8_t*)ref->data, excl_mask_ref, part, ref->nz, ref->ny, ref->nx);
      break;
    default:
      k_penalty_partial<float><<<nblk, kThreads, 0, s>>>((const float*)ref->data, excl_mask_ref, part, ref->nz, ref->ny, ref->nx);
  }
  k_penalty_final<<<1, 1024, 0, s>>>(part, nblk, factor_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "wr_penalty_factor_noalloc launch");
  return WR_OK;
}

int wr_resize_table(int32_t in_len, int32_t out_len, int32_t method, double* weights, int32_t* indices,
                    int32_t* taps) {
  if (!taps) return fail(WR_E_NULL, "taps is NULL");
  if (in_len < 1 || out_len < 1) return fail(WR_E_SHAPE, "lengths must be positive");
  if (method != RESIZE_BICUBIC && method != RESIZE_BILINEAR) return fail(WR_E_PARAM, "method must be 0 or 1");
  int P = resize_taps(in_len, out_len);
  *taps = P;
  if (!weights) return WR_OK;
  if (!indices) return fail(WR_E_NULL, "indices is NULL");
  for (int k = 0; k < out_len; ++k)
    resize_row(in_len, out_len, method, k, weights + (size_t)k * P, indices + (size_t)k * P);
  return WR_OK;
}

}  // extern "C"
