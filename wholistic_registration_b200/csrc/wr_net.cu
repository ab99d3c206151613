// Kernels of the learned warm-start network: a small 3-D convolutional
// encoder-decoder that predicts a coarse displacement field (1/4 resolution in
// x and y) from a template / moving pair.  No counterpart exists in the
// reference; its output enters the registration through the reference's own
// warm-start channel, option["motion"] (utils/calFlow3d_Wei_v1.py:362-377).
//
// Tensors are channels-last bfloat16: [n][z][y][x][c], channel counts padded
// to multiples of 16.  A convolution is an implicit GEMM on the tcgen05 BF16
// tensor cores, float32 accumulators in tensor memory (wr_net_tc_conv.inc):
//   forward  y[q][co] = act(b[co] + sum_{tap,ci} x[p(q,tap)][ci] w[tap][co][ci])
//   data     dx[p][ci] = sum_{tap,co} dy[q(p,tap)][co] w[tap][co][ci]
//   weights  dw[tap][co][ci] = sum_q dy[q][co] x[p(q,tap)][ci]
// with p = stride*q + tap - 1 per axis (3x3x3 kernel, padding 1).  The input
// of a decoder convolution is the virtual concatenation of a coarser tensor
// (nearest-upsampled by 2: its voxel is p/2) and a skip tensor; the gather
// reads either directly, so no upsampled or concatenated copy is formed.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "wr_b200.h"
#include "wr_net.h"
#include "wr_net_tc.cuh"

namespace wrnet {

static thread_local std::string g_err;

static int fail(int code, const char* m) {
  g_err = m;
  return code;
}

static int cuda_status(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return WR_OK;
  g_err = std::string(where) + ": " + cudaGetErrorString(e);
  return -(int)e;
}


// Geometry of one convolution (all extents of the output / input grids).
struct Conv {
  int n;                // batch
  int oz, oy, ox;       // output grid
  int iz, iy, ix;       // input grid (of the skip / direct source)
  int stride;           // 1 or 2
  int c1, c2;           // channels from source 1 and source 2 (c2 = 0: single source)
  int up1;              // source 1 is half resolution, read at p / 2
  int cin;              // c1 + c2 (multiple of 16)
  int cout;             // real output channels
  int cout_p;           // padded to a multiple of 16 (weight rows)
  int act;              // 1: LeakyReLU(0.1)
};

__device__ __forceinline__ long long vox(int n, int z, int y, int x, int Z, int Y, int X) {
  return (((long long)n * Z + z) * Y + y) * X + x;
}

#include "wr_net_tc_conv.inc"

__global__ void k_act_backward(const float* __restrict__ grad, const __nv_bfloat16* __restrict__ y, int act,
                               __nv_bfloat16* __restrict__ dpre, long long nvox, int cout, int cout_p) {
  const long long total = nvox * cout_p;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long v = i / cout_p;
    const int co = (int)(i - v * cout_p);
    float d = 0.f;
    if (co < cout) {
      d = grad[v * cout + co];
      if (act && y != nullptr && __bfloat162float(y[v * cout + co]) <= 0.f) d *= 0.1f;
    }
    dpre[i] = __float2bfloat16(d);
  }
}

// scatter the virtual input's gradient: channels [0, c1) go to source 1
// (summed over the 2x2x2 fine voxels of each coarse voxel when upsampled),
// channels [c1, cin) to source 2; both accumulate (+=)
__global__ void k_split_grad(Conv c, const float* __restrict__ dxv, float* __restrict__ g1, float* __restrict__ g2) {
  const long long nvox = (long long)c.n * c.iz * c.iy * c.ix;
  const long long total = nvox * c.cin;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long p = i / c.cin;
    const int ch = (int)(i - p * c.cin);
    const float v = dxv[i];
    if (ch >= c.c1) {
      if (g2) g2[p * c.c2 + (ch - c.c1)] += v;
    } else if (g1) {
      if (c.up1) {
        long long pp = p;
        const int x = (int)(pp % c.ix); pp /= c.ix;
        const int y = (int)(pp % c.iy); pp /= c.iy;
        const int z = (int)(pp % c.iz); const int n = (int)(pp / c.iz);
        const long long q = vox(n, z >> 1, y >> 1, x >> 1, (c.iz + 1) / 2, (c.iy + 1) / 2, (c.ix + 1) / 2);
        atomicAdd(g1 + q * c.c1 + ch, v);
      } else {
        g1[p * c.c1 + ch] += v;
      }
    }
  }
}

// Adam on float32 master weights; also writes the bf16 forward weights and,
// for layers with a data-gradient pass, the transposed bf16 weights
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ gw, float* __restrict__ m, float* __restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2, float decay) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = gw[i] + decay * w[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// float32 [tap][cout_p][cin] -> bf16 forward weights and bf16 [tap][cin][cout_p]
__global__ void k_weights_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wf,
                                  __nv_bfloat16* __restrict__ wt, int cout_p, int cin) {
  const long long n = 27LL * cout_p * cin;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long tap = i / ((long long)cout_p * cin);
    const int rem = (int)(i - tap * cout_p * cin);
    const int co = rem / cin, ci = rem - co * cin;
    const __nv_bfloat16 b = __float2bfloat16(w[i]);
    wf[i] = b;
    if (wt) wt[(tap * cin + ci) * cout_p + co] = b;
  }
}

// flow loss: l2 * mean |pred - target|^2 plus a warped-residual term
// res * mean (mov(p + f(p)) - tmpl(p))^2 on the network's grid (flow in
// full-resolution voxels; x and y are divided by `scale` on that grid)
__global__ void k_flow_loss(const float* __restrict__ pred, const float* __restrict__ target,
                            const float* __restrict__ tmpl, const float* __restrict__ mov, float* __restrict__ grad,
                            double* __restrict__ loss, int n, int Z, int Y, int X, float scale, float l2, float res) {
  const long long nvox = (long long)n * Z * Y * X;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvox;
       i += (long long)gridDim.x * blockDim.x) {
    float g[3] = {0.f, 0.f, 0.f};
    double li = 0.0;
    for (int k = 0; k < 3; ++k) {
      const float d = pred[3 * i + k] - target[3 * i + k];
      li += (double)l2 * d * d;
      g[k] = 2.f * l2 * d;
    }
    if (res > 0.f) {
      long long ii = i;
      const int x = (int)(ii % X); ii /= X;
      const int y = (int)(ii % Y); ii /= Y;
      const int z = (int)(ii % Z); const int b = (int)(ii / Z);
      const float cx = x + pred[3 * i] / scale, cy = y + pred[3 * i + 1] / scale, cz = z + pred[3 * i + 2];
      const float fx = floorf(cx), fy = floorf(cy), fz = floorf(cz);
      const float tx = cx - fx, ty = cy - fy, tz = cz - fz;
      int xs[2], ys[2], zs[2];
      xs[0] = min(max((int)fx, 0), X - 1); xs[1] = min(max((int)fx + 1, 0), X - 1);
      ys[0] = min(max((int)fy, 0), Y - 1); ys[1] = min(max((int)fy + 1, 0), Y - 1);
      zs[0] = min(max((int)fz, 0), Z - 1); zs[1] = min(max((int)fz + 1, 0), Z - 1);
      float v = 0.f, dvx = 0.f, dvy = 0.f, dvz = 0.f;
      for (int a = 0; a < 2; ++a)
        for (int bb = 0; bb < 2; ++bb)
          for (int cc = 0; cc < 2; ++cc) {
            const float m = mov[(((long long)b * Z + zs[a]) * Y + ys[bb]) * X + xs[cc]];
            const float wz = a ? tz : 1.f - tz, wy = bb ? ty : 1.f - ty, wx = cc ? tx : 1.f - tx;
            v += wz * wy * wx * m;
            dvx += wz * wy * (cc ? 1.f : -1.f) * m;
            dvy += wz * wx * (bb ? 1.f : -1.f) * m;
            dvz += wy * wx * (a ? 1.f : -1.f) * m;
          }
      const float r = v - tmpl[i];
      li += (double)res * r * r;
      g[0] += 2.f * res * r * dvx / scale;
      g[1] += 2.f * res * r * dvy / scale;
      g[2] += 2.f * res * r * dvz;
    }
    for (int k = 0; k < 3; ++k) grad[3 * i + k] = g[k] / (float)nvox;
    acc += li;
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] / (double)nvox);
}

// mean of a (z, y, x) volume (float64), one value to device memory
template <typename T>
__global__ void k_mean(const T* __restrict__ v, long long n, double* __restrict__ out) {
  __shared__ double red[256];
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    acc += (double)v[i];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, red[0] / (double)n);
}

// network input: f x f mean pooling in x and y of template (channel 0) and
// moving (channel 1), divided by the template mean; channels 2..15 zero.
// Float32 copies of both pooled volumes feed the residual loss.
template <typename T>
__global__ void k_pool_input(const T* __restrict__ tmpl, const T* __restrict__ mov, const double* __restrict__ mean,
                             int Z, int Y, int X, int f, __nv_bfloat16* __restrict__ x0, float* __restrict__ t4,
                             float* __restrict__ m4) {
  const int Yq = Y / f, Xq = X / f;
  const long long n = (long long)Z * Yq * Xq;
  const float inv = (float)(1.0 / fmax(*mean, 1e-12));
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % Xq);
    const long long r = i / Xq;
    const int y = (int)(r % Yq), z = (int)(r / Yq);
    float st = 0.f, sm = 0.f;
    for (int dy = 0; dy < f; ++dy)
      for (int dx = 0; dx < f; ++dx) {
        const long long p = ((long long)z * Y + y * f + dy) * X + x * f + dx;
        st += (float)tmpl[p];
        sm += (float)mov[p];
      }
    st *= inv / (f * f);
    sm *= inv / (f * f);
    if (t4) t4[i] = st;
    if (m4) m4[i] = sm;
    __nv_bfloat16* o = x0 + i * 16;
    o[0] = __float2bfloat16(st);
    o[1] = __float2bfloat16(sm);
    for (int c = 2; c < 16; ++c) o[c] = __float2bfloat16(0.f);
  }
}

// flow (z, y, x, 3) -> mean over f x f blocks in x and y
__global__ void k_pool_flow(const float* __restrict__ flow, int Z, int Y, int X, int f, float* __restrict__ out) {
  const int Yq = Y / f, Xq = X / f;
  const long long n = (long long)Z * Yq * Xq;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % Xq);
    const long long r = i / Xq;
    const int y = (int)(r % Yq), z = (int)(r / Yq);
    float a[3] = {0.f, 0.f, 0.f};
    for (int dy = 0; dy < f; ++dy)
      for (int dx = 0; dx < f; ++dx) {
        const long long p = ((long long)z * Y + y * f + dy) * X + x * f + dx;
        for (int c = 0; c < 3; ++c) a[c] += flow[3 * p + c];
      }
    for (int c = 0; c < 3; ++c) out[3 * i + c] = a[c] / (f * f);
  }
}

// coarse flow (z, Y/f, X/f, 3) -> full-resolution (z, Y, X, 3), bilinear in x
// and y on pixel centres, edge-clamped
__global__ void k_upsample_flow(const float* __restrict__ fq, int Z, int Y, int X, int f, float* __restrict__ out) {
  const int Yq = Y / f, Xq = X / f;
  const long long n = (long long)Z * Y * X;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % X);
    const long long r = i / X;
    const int y = (int)(r % Y), z = (int)(r / Y);
    const float cx = fminf(fmaxf((x + 0.5f) / f - 0.5f, 0.f), (float)(Xq - 1));
    const float cy = fminf(fmaxf((y + 0.5f) / f - 0.5f, 0.f), (float)(Yq - 1));
    const int x0 = (int)cx, y0 = (int)cy;
    const int x1 = min(x0 + 1, Xq - 1), y1 = min(y0 + 1, Yq - 1);
    const float tx = cx - x0, ty = cy - y0;
    const float* b = fq + (long long)z * Yq * Xq * 3;
    for (int c = 0; c < 3; ++c) {
      const float v00 = b[(y0 * Xq + x0) * 3 + c], v01 = b[(y0 * Xq + x1) * 3 + c];
      const float v10 = b[(y1 * Xq + x0) * 3 + c], v11 = b[(y1 * Xq + x1) * 3 + c];
      out[3 * i + c] = (1.f - ty) * ((1.f - tx) * v00 + tx * v01) + ty * ((1.f - tx) * v10 + tx * v11);
    }
  }
}

// mean of (a - b)^2 over voxels not excluded (mask == 0 or no mask)
template <typename T>
__global__ void k_masked_mse(const float* __restrict__ a, const T* __restrict__ b, const uint8_t* __restrict__ excl,
                             long long n, double* __restrict__ out) {
  __shared__ double red[2][256];
  double s = 0.0, c = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (excl && excl[i]) continue;
    const double d = (double)a[i] - (double)b[i];
    s += d * d;
    c += 1.0;
  }
  red[0][threadIdx.x] = s;
  red[1][threadIdx.x] = c;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) {
      red[0][threadIdx.x] += red[0][threadIdx.x + k];
      red[1][threadIdx.x] += red[1][threadIdx.x + k];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    atomicAdd(out, red[0][0]);
    atomicAdd(out + 1, red[1][0]);
  }
}

static int grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b < 1) b = 1;
  return (int)(b < 148LL * 16 ? b : 148LL * 16);
}

static int check(const WrConvGeom* g, Conv* c) {
  if (!g) return fail(WR_E_NULL, "geometry is NULL");
  c->n = g->n; c->oz = g->oz; c->oy = g->oy; c->ox = g->ox;
  c->iz = g->iz; c->iy = g->iy; c->ix = g->ix;
  c->stride = g->stride; c->c1 = g->c1; c->c2 = g->c2; c->up1 = g->up1;
  c->cin = g->c1 + g->c2; c->cout = g->cout; c->cout_p = (g->cout + 15) / 16 * 16; c->act = g->act;
  if (c->n < 1 || c->oz < 1 || c->oy < 1 || c->ox < 1 || c->iz < 1 || c->iy < 1 || c->ix < 1)
    return fail(WR_E_SHAPE, "empty grid");
  if (c->stride != 1 && c->stride != 2) return fail(WR_E_PARAM, "stride must be 1 or 2");
  if (c->c1 % 16 || c->c2 % 16 || c->cin < 16 || c->cin > 112) return fail(WR_E_PARAM, "channels must be multiples of 16, total <= 112");
  if (c->cout < 1 || c->cout_p > 64) return fail(WR_E_PARAM, "cout must be in [1, 64]");
  const int ez = (c->iz - 1) / c->stride + 1, ey = (c->iy - 1) / c->stride + 1, ex = (c->ix - 1) / c->stride + 1;
  if (c->oz != ez || c->oy != ey || c->ox != ex) return fail(WR_E_SHAPE, "output grid does not match input and stride");
  return WR_OK;
}

// flag the tcgen05 kernels set when a wait runs out (one per device)
static __device__ int g_tc_err;

static int* tc_err_ptr() {
  static std::mutex mu;
  static int* ptr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_tc_err) != cudaSuccess) return nullptr;
    ptr[dev] = static_cast<int*>(p);
  }
  return ptr[dev];
}

template <int MODE, int NT>
static int launch_tc(const Conv& c, long long rows, int kc, const void* x1, const void* x2, const void* w,
                     const float* b, void* y, float* y32, float* dx, cudaStream_t s) {
  int* err = tc_err_ptr();
  if (!err) return fail(WR_E_PARAM, "no CUDA device for the tensor-core convolution");
  const size_t smem = tc_smem_bytes(kc, 16 * NT);
  cudaFuncSetAttribute(k_conv_tc<MODE, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const unsigned blocks = (unsigned)((rows + kTcRows - 1) / kTcRows);
  k_conv_tc<MODE, NT><<<blocks, kTcThreads, smem, s>>>(c, (const __nv_bfloat16*)x1, (const __nv_bfloat16*)x2,
                                                       (const __nv_bfloat16*)w, b, (__nv_bfloat16*)y, y32, dx, err);
  return WR_OK;
}

template <int NT>
static int launch_wgrad_tc(const Conv& c, const void* x1, const void* x2, const void* dy, float* dw, float* db,
                           cudaStream_t s) {
  int* err = tc_err_ptr();
  if (!err) return fail(WR_E_PARAM, "no CUDA device for the tensor-core convolution");
  const size_t smem = tc_wgrad_smem_bytes(16 * NT);
  cudaFuncSetAttribute(k_conv_wgrad_tc<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const long long nvox = (long long)c.n * c.oz * c.oy * c.ox;
  const dim3 grid((unsigned)((nvox + kWgK * kWgStages - 1) / (kWgK * kWgStages)), 27);
  k_conv_wgrad_tc<NT><<<grid, kTcThreads, smem, s>>>(c, (const __nv_bfloat16*)x1, (const __nv_bfloat16*)x2,
                                                     (const __nv_bfloat16*)dy, dw, db, err);
  return WR_OK;
}

}  // namespace wrnet

using namespace wrnet;

extern "C" {

const char* wr_net_last_error(void) { return g_err.c_str(); }

int wr_net_tc_error(int* flag) {
  if (!flag) return fail(WR_E_NULL, "flag is NULL");
  int* p = tc_err_ptr();
  if (!p) return fail(WR_E_PARAM, "no CUDA device");
  int v = 0;
  cudaError_t e = cudaMemcpy(&v, p, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemset(p, 0, sizeof(int));
  if (e != cudaSuccess) return cuda_status("wr_net_tc_error");
  *flag = v;
  return WR_OK;
}

int wr_net_conv3d_fwd(const WrConvGeom* geom, const void* x1, const void* x2, const void* w, const float* bias,
                      void* y, float* y32, void* stream) {
  Conv c;
  int rc = check(geom, &c);
  if (rc) return rc;
  if (!x1 || !w || !bias || (!y && !y32) || (c.c2 && !x2)) return fail(WR_E_NULL, "a required pointer is NULL");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long rows = (long long)c.n * c.oz * c.oy * c.ox;
  switch (c.cout_p / 16) {
    case 1: rc = launch_tc<kTcFwd, 1>(c, rows, c.cin, x1, x2, w, bias, y, y32, nullptr, s); break;
    case 2: rc = launch_tc<kTcFwd, 2>(c, rows, c.cin, x1, x2, w, bias, y, y32, nullptr, s); break;
    case 3: rc = launch_tc<kTcFwd, 3>(c, rows, c.cin, x1, x2, w, bias, y, y32, nullptr, s); break;
    default: rc = launch_tc<kTcFwd, 4>(c, rows, c.cin, x1, x2, w, bias, y, y32, nullptr, s); break;
  }
  if (rc) return rc;
  return cuda_status("wr_net_conv3d_fwd");
}

int wr_net_conv3d_dgrad(const WrConvGeom* geom, const void* dy, const void* wt, float* dxv, void* stream) {
  Conv c;
  int rc = check(geom, &c);
  if (rc) return rc;
  if (!dy || !wt || !dxv) return fail(WR_E_NULL, "a required pointer is NULL");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long rows = (long long)c.n * c.iz * c.iy * c.ix;
  switch (c.cin / 16) {
    case 1: rc = launch_tc<kTcDgrad, 1>(c, rows, c.cout_p, dy, nullptr, wt, nullptr, nullptr, nullptr, dxv, s); break;
    case 2: rc = launch_tc<kTcDgrad, 2>(c, rows, c.cout_p, dy, nullptr, wt, nullptr, nullptr, nullptr, dxv, s); break;
    case 3: rc = launch_tc<kTcDgrad, 3>(c, rows, c.cout_p, dy, nullptr, wt, nullptr, nullptr, nullptr, dxv, s); break;
    case 4: rc = launch_tc<kTcDgrad, 4>(c, rows, c.cout_p, dy, nullptr, wt, nullptr, nullptr, nullptr, dxv, s); break;
    case 5: rc = launch_tc<kTcDgrad, 5>(c, rows, c.cout_p, dy, nullptr, wt, nullptr, nullptr, nullptr, dxv, s); break;
    case 6: rc = launch_tc<kTcDgrad, 6>(c, rows, c.cout_p, dy, nullptr, wt, nullptr, nullptr, nullptr, dxv, s); break;
    default: rc = launch_tc<kTcDgrad, 7>(c, rows, c.cout_p, dy, nullptr, wt, nullptr, nullptr, nullptr, dxv, s); break;
  }
  if (rc) return rc;
  return cuda_status("wr_net_conv3d_dgrad");
}

int wr_net_conv3d_wgrad(const WrConvGeom* geom, const void* x1, const void* x2, const void* dy, float* dw, float* db,
                        void* stream) {
  Conv c;
  int rc = check(geom, &c);
  if (rc) return rc;
  if (!x1 || !dy || !dw || (c.c2 && !x2)) return fail(WR_E_NULL, "a required pointer is NULL");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (c.cout_p / 16) {
    case 1: rc = launch_wgrad_tc<1>(c, x1, x2, dy, dw, db, s); break;
    case 2: rc = launch_wgrad_tc<2>(c, x1, x2, dy, dw, db, s); break;
    case 3: rc = launch_wgrad_tc<3>(c, x1, x2, dy, dw, db, s); break;
    default: rc = launch_wgrad_tc<4>(c, x1, x2, dy, dw, db, s); break;
  }
  if (rc) return rc;
  return cuda_status("wr_net_conv3d_wgrad");
}

int wr_net_act_backward(const float* grad, const void* y, int act, void* dpre, long long nvox, int cout, void* stream) {
  if (!grad || !dpre) return fail(WR_E_NULL, "a required pointer is NULL");
  const int cout_p = (cout + 15) / 16 * 16;
  k_act_backward<<<grid_for(nvox * cout_p), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      grad, (const __nv_bfloat16*)y, act, (__nv_bfloat16*)dpre, nvox, cout, cout_p);
  return cuda_status("wr_net_act_backward");
}

int wr_net_split_grad(const WrConvGeom* geom, const float* dxv, float* g1, float* g2, void* stream) {
  Conv c;
  int rc = check(geom, &c);
  if (rc) return rc;
  if (!dxv) return fail(WR_E_NULL, "dxv is NULL");
  const long long nvox = (long long)c.n * c.iz * c.iy * c.ix;
  k_split_grad<<<grid_for(nvox * c.cin), 256, 0, static_cast<cudaStream_t>(stream)>>>(c, dxv, g1, g2);
  return cuda_status("wr_net_split_grad");
}

int wr_net_adam(float* w, const float* gw, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
                int step, float decay, void* stream) {
  if (!w || !gw || !m || !v) return fail(WR_E_NULL, "a required pointer is NULL");
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(w, gw, m, v, n, lr, b1, b2, eps, c1, c2, decay);
  return cuda_status("wr_net_adam");
}

int wr_net_weights_to_bf16(const float* w, void* wf, void* wt, int cout, int cin, void* stream) {
  if (!w || !wf) return fail(WR_E_NULL, "a required pointer is NULL");
  const int cout_p = (cout + 15) / 16 * 16;
  k_weights_to_bf16<<<grid_for(27LL * cout_p * cin), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      w, (__nv_bfloat16*)wf, (__nv_bfloat16*)wt, cout_p, cin);
  return cuda_status("wr_net_weights_to_bf16");
}

int wr_net_flow_loss(const float* pred, const float* target, const float* tmpl, const float* mov, float* grad,
                     double* loss, int n, int nz, int ny, int nx, float scale, float l2, float res, void* stream) {
  if (!pred || !target || !grad || !loss || (res > 0.f && (!tmpl || !mov))) return fail(WR_E_NULL, "a required pointer is NULL");
  k_flow_loss<<<grid_for((long long)n * nz * ny * nx), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      pred, target, tmpl, mov, grad, loss, n, nz, ny, nx, scale, l2, res);
  return cuda_status("wr_net_flow_loss");
}

int wr_net_prepare_input(const WrVolume* tmpl, const WrVolume* mov, int factor, double* mean_scratch, void* x0,
                         float* t4, float* m4, void* stream) {
  if (!tmpl || !mov || !tmpl->data || !mov->data || !mean_scratch || !x0) return fail(WR_E_NULL, "a required pointer is NULL");
  if (tmpl->dtype != mov->dtype || (tmpl->dtype != WR_U16 && tmpl->dtype != WR_F32)) return fail(WR_E_DTYPE, "uint16 or float32 volumes of one type");
  if (tmpl->nz != mov->nz || tmpl->ny != mov->ny || tmpl->nx != mov->nx) return fail(WR_E_SHAPE, "shapes differ");
  if (factor < 1 || tmpl->ny % factor || tmpl->nx % factor) return fail(WR_E_SHAPE, "x and y extents must be multiples of factor");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long n = (long long)tmpl->nz * tmpl->ny * tmpl->nx;
  const long long nq = n / (factor * factor);
  cudaMemsetAsync(mean_scratch, 0, sizeof(double), s);
  if (tmpl->dtype == WR_U16) {
    k_mean<uint16_t><<<grid_for(n), 256, 0, s>>>((const uint16_t*)tmpl->data, n, mean_scratch);
    k_pool_input<uint16_t><<<grid_for(nq), 256, 0, s>>>((const uint16_t*)tmpl->data, (const uint16_t*)mov->data,
                                                        mean_scratch, tmpl->nz, tmpl->ny, tmpl->nx, factor,
                                                        (__nv_bfloat16*)x0, t4, m4);
  } else {
    k_mean<float><<<grid_for(n), 256, 0, s>>>((const float*)tmpl->data, n, mean_scratch);
    k_pool_input<float><<<grid_for(nq), 256, 0, s>>>((const float*)tmpl->data, (const float*)mov->data, mean_scratch,
                                                     tmpl->nz, tmpl->ny, tmpl->nx, factor, (__nv_bfloat16*)x0, t4, m4);
  }
  return cuda_status("wr_net_prepare_input");
}

int wr_net_masked_sse(const float* a, const WrVolume* b, const uint8_t* excl, double* out2, void* stream) {
  if (!a || !b || !b->data || !out2) return fail(WR_E_NULL, "a required pointer is NULL");
  const long long n = (long long)b->nz * b->ny * b->nx;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (b->dtype == WR_U16) k_masked_mse<uint16_t><<<grid_for(n), 256, 0, s>>>(a, (const uint16_t*)b->data, excl, n, out2);
  else if (b->dtype == WR_F32) k_masked_mse<float><<<grid_for(n), 256, 0, s>>>(a, (const float*)b->data, excl, n, out2);
  else return fail(WR_E_DTYPE, "uint16 or float32 volume");
  return cuda_status("wr_net_masked_sse");
}

int wr_net_pool_flow(const float* flow, int nz, int ny, int nx, int factor, float* out, void* stream) {
  if (!flow || !out) return fail(WR_E_NULL, "a required pointer is NULL");
  if (factor < 1 || ny % factor || nx % factor) return fail(WR_E_SHAPE, "x and y extents must be multiples of factor");
  const long long nq = (long long)nz * (ny / factor) * (nx / factor);
  k_pool_flow<<<grid_for(nq), 256, 0, static_cast<cudaStream_t>(stream)>>>(flow, nz, ny, nx, factor, out);
  return cuda_status("wr_net_pool_flow");
}

int wr_net_upsample_flow(const float* fq, int nz, int ny, int nx, int factor, float* out, void* stream) {
  if (!fq || !out) return fail(WR_E_NULL, "a required pointer is NULL");
  if (factor < 1 || ny % factor || nx % factor) return fail(WR_E_SHAPE, "x and y extents must be multiples of factor");
  k_upsample_flow<<<grid_for((long long)nz * ny * nx), 256, 0, static_cast<cudaStream_t>(stream)>>>(fq, nz, ny, nx,
                                                                                                     factor, out);
  return cuda_status("wr_net_upsample_flow");
}

}  // extern "C"
