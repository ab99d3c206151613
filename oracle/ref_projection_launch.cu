// Test infrastructure, not product code: host launchers for the reference's
// two projection kernels, whose CUDA C source is embedded as strings in
// src/wholistic_registration/utils/calFlowCrossResolution.py
// (project_to_planes_nanmax_kernel :480-569, project_to_planes_weighted_avg_kernel
// :571-660).  oracle/build_ref_projection.py extracts that source unchanged
// into oracle/_ref/ref_projection_kernels.cu and compiles it with this file;
// the launch shape is the reference wrappers' (256 threads, one thread per
// (sample, plane) pair, :834 and :1089).  The fixtures made with it pin the
// oracle's and the library's projections to the reference's own kernels.
#include <cuda_runtime.h>

#include "ref_projection_kernels.cu"

extern "C" int ref_project_nanmax_launch(const float* values, const float* coords, const float* target_z, float* out,
                                         long long nvox, int nplanes, int xref, int yref, int xout, int yout,
                                         float z_window, int downsample_xy, int use_nearest_xy, int xy_extra_radius) {
  const int threads = 256;
  const long long blocks = (nvox * nplanes + threads - 1) / threads;
  if (blocks <= 0) return 0;
  project_to_planes_nanmax_kernel<<<(unsigned)blocks, threads>>>(values, coords, target_z, out, nvox, nplanes, xref,
                                                                   yref, xout, yout, z_window, downsample_xy,
                                                                   use_nearest_xy, xy_extra_radius);
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? (int)cudaGetLastError() : (int)e;
}

extern "C" int ref_project_weighted_launch(const float* values, const float* coords, const float* target_z,
                                           float* sum_val, float* sum_w, long long nvox, int nplanes, int xref,
                                           int yref, int xout, int yout, float z_window, float z_sigma,
                                           int downsample_xy, int z_weight_mode) {
  const int threads = 256;
  const long long blocks = (nvox * nplanes + threads - 1) / threads;
  if (blocks <= 0) return 0;
  project_to_planes_weighted_avg_kernel<<<(unsigned)blocks, threads>>>(values, coords, target_z, sum_val, sum_w, nvox,
                                                                         nplanes, xref, yref, xout, yout, z_window,
                                                                         z_sigma, downsample_xy, z_weight_mode);
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? (int)cudaGetLastError() : (int)e;
}
