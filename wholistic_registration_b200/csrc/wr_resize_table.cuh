// Resize tap tables (MATLAB imresize semantics), computed identically on the
// host and on the device.
//
// Restates utils/imresize.py:41-82 (triangle, cubic, contributions).  The
// float64 arithmetic is written operation by operation with explicit
// round-to-nearest intrinsics on the device (no fused multiply-add), and the
// row normalisation reproduces NumPy's pairwise summation, so the tables equal
// the reference's float64 tables bit for bit.  That exactness matters for the
// exclusion masks, whose resized values are thresholded at > 0
// (utils/calFlow3d_Wei_v1.py:422-423,473).
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define WR_HD __host__ __device__
#else
#define WR_HD
#endif

namespace wr {

#if defined(__CUDA_ARCH__)
WR_HD inline double dmul(double a, double b) { return __dmul_rn(a, b); }
WR_HD inline double dadd(double a, double b) { return __dadd_rn(a, b); }
WR_HD inline double dsub(double a, double b) { return __dsub_rn(a, b); }
WR_HD inline double ddiv(double a, double b) { return __ddiv_rn(a, b); }
#else
// host code is compiled with -ffp-contract=off
WR_HD inline double dmul(double a, double b) { return a * b; }
WR_HD inline double dadd(double a, double b) { return a + b; }
WR_HD inline double dsub(double a, double b) { return a - b; }
WR_HD inline double ddiv(double a, double b) { return a / b; }
#endif

// Keys cubic, a = -0.5 (utils/imresize.py:49-57), same operation order.
WR_HD inline double cubic_kernel(double t) {
  double a = fabs(t);
  double a2 = dmul(a, a);
  double a3 = dmul(a2, a);
  double near = dadd(dsub(dmul(1.5, a3), dmul(2.5, a2)), 1.0);
  double far = dadd(dsub(dadd(dmul(-0.5, a3), dmul(2.5, a2)), dmul(4.0, a)), 2.0);
  double f1 = (a <= 1.0) ? near : 0.0;
  double f2 = (a > 1.0 && a <= 2.0) ? far : 0.0;
  // the reference multiplies each branch by a 0/1 mask and adds them
  return dadd(dmul(f1, 1.0), dmul(f2, 1.0));
}

// Tent kernel (utils/imresize.py:41-46).
WR_HD inline double triangle_kernel(double t) {
  double left = (t >= -1.0 && t < 0.0) ? dadd(t, 1.0) : 0.0;
  double right = (t <= 1.0 && t >= 0.0) ? dsub(1.0, t) : 0.0;
  return dadd(left, right);
}

// NumPy's pairwise sum of a contiguous float64 row (8 accumulators for
// 8 <= n <= 128, recursive halving above).
WR_HD inline double np_pairwise_sum(const double* a, int n) {
  if (n < 8) {
    double res = -0.0;
    for (int i = 0; i < n; ++i) res = dadd(res, a[i]);
    return res;
  }
  if (n <= 128) {
    double r0 = a[0], r1 = a[1], r2 = a[2], r3 = a[3];
    double r4 = a[4], r5 = a[5], r6 = a[6], r7 = a[7];
    int i = 8;
    for (; i < n - (n % 8); i += 8) {
      r0 = dadd(r0, a[i + 0]); r1 = dadd(r1, a[i + 1]);
      r2 = dadd(r2, a[i + 2]); r3 = dadd(r3, a[i + 3]);
      r4 = dadd(r4, a[i + 4]); r5 = dadd(r5, a[i + 5]);
      r6 = dadd(r6, a[i + 6]); r7 = dadd(r7, a[i + 7]);
    }
    double res = dadd(dadd(dadd(r0, r1), dadd(r2, r3)), dadd(dadd(r4, r5), dadd(r6, r7)));
    for (; i < n; ++i) res = dadd(res, a[i]);
    return res;
  }
  int n2 = n / 2;
  n2 -= n2 % 8;
  return dadd(np_pairwise_sum(a, n2), np_pairwise_sum(a + n2, n - n2));
}

enum { RESIZE_BICUBIC = 0, RESIZE_BILINEAR = 1 };

// Scale the reference derives from the shapes (utils/imresize.py:34-38).
WR_HD inline double resize_scale(int in_len, int out_len) {
  return ddiv(dmul(1.0, (double)out_len), (double)in_len);
}

// Number of candidate taps per output, P = ceil(width) + 2.
WR_HD inline int resize_taps(int in_len, int out_len) {
  double scale = resize_scale(in_len, out_len);
  double width = scale < 1.0 ? ddiv(dmul(1.0, 4.0), scale) : 4.0;
  return (int)ceil(width) + 2;
}

// One row of contributions(): weights[t], indices[t] for output k (0-based),
// t = 0..P-1, before the reference drops all-zero columns (dropping them does
// not change any weighted sum).  Returns P.
WR_HD inline int resize_row(int in_len, int out_len, int method, int k, double* weights,
                            int32_t* indices) {
  double scale = resize_scale(in_len, out_len);
  bool shrink = scale < 1.0;
  double width = shrink ? ddiv(dmul(1.0, 4.0), scale) : 4.0;
  int P = (int)ceil(width) + 2;
  double x = (double)(k + 1);
  double u = dadd(ddiv(x, scale), dmul(0.5, dsub(1.0, ddiv(1.0, scale))));
  double left = floor(dsub(u, ddiv(width, 2.0)));
  for (int t = 0; t < P; ++t) {
    int32_t ind = (int32_t)dsub(dadd(left, (double)t), 1.0);
    double arg = dsub(dsub(u, (double)ind), 1.0);
    double w;
    if (method == RESIZE_BICUBIC) {
      w = shrink ? dmul(scale, cubic_kernel(dmul(scale, arg))) : cubic_kernel(arg);
    } else {
      w = shrink ? dmul(scale, triangle_kernel(dmul(scale, arg))) : triangle_kernel(arg);
    }
    weights[t] = w;
    // symmetric reflection: aux = [0..n-1, n-1..0], index mod 2n
    int m = 2 * in_len;
    int j = ind % m;
    if (j < 0) j += m;
    indices[t] = j < in_len ? j : (m - 1 - j);
  }
  double s = np_pairwise_sum(weights, P);
  for (int t = 0; t < P; ++t) weights[t] = ddiv(weights[t], s);
  return P;
}

}  // namespace wr
