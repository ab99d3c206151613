/*
 * wr_xres.h - C ABI of the cross-resolution registration (getMotion_v2).
 *
 * Replaces the reference entry point (path relative to src/wholistic_registration/)
 *
 *   wr_xres_register   utils/calFlowCrossResolution.py:2470-2663
 *                      getMotion_v2(data_mov, data_ref, option)
 *
 * The moving stack lives on the iteration grid, the reference stack on its own
 * grid (another z spacing, possibly other x / y extents); the reference is
 * read through its cubic B-spline (map_coordinates order 3, mode "nearest")
 * at the phase p = (x, y, z zRatio / zRatio_HR) + motion.
 *
 * Layouts are the (z, y, x) memory order of the reference's (x, y, z) arrays:
 * volumes (nz, ny, nx) float32, fields (nz, ny, nx, 3) float32 with component
 * 0 along x.  All pointers are device pointers on the caller's stream.
 */
#ifndef WR_XRES_H
#define WR_XRES_H

#include "wr_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * getMotion_v2's wrong-region correction (utils/calFlowCrossResolution.py:
 * 2240-2467, option keys in brackets): after each layer's optimisation, CPs
 * whose local error is a robust outlier are grouped into regions, their
 * voxels' phases seed a trap mask in reference space, and the layer is
 * re-run with the trap excluded and then refined with the original masks;
 * the refined result is kept when its error is lower.  enable = 0: off.
 */
typedef struct WrXresWrongRegion {
  int32_t enable;              /* ["wrong_region_enable"] */
  int32_t metric;              /* ["wrong_region_metric"]: 0 "mse", 1 "mae" */
  float mad_threshold;         /* ["wrong_region_mad_threshold"], 3.0 */
  int32_t min_component_size;  /* ["wrong_region_min_component_size"], 2 */
  float expand_radius_xy;      /* ["expand_radius_xy"], 2.0 (divided by 2^layer) */
  float sigma_grad;            /* ["sigma_grad"], 1.0 */
  float intensity_k;           /* ["intensity_k"], 2.0 */
  int32_t exclude_mode;        /* ["wrong_region_exclude_mode"]: 0 "direct", 1 "highresidual" (only the bad
                                  voxels whose 3x3-smoothed error drop over the pass reaches the quantile below
                                  seed the trap, :2340-2355) */
  float quantile_q;            /* ["quantile_threshold_q"], 0.8 */
} WrXresWrongRegion;

/*
 * Workspace bytes for a moving stack (nz, ny, nx) and a reference stack
 * (nzh, nyh, nxh).  p->precision must be WR_PREC_F32; p->zRatio is the
 * moving stack's z spacing (option["zRatio"]), zRatio_HR the reference's
 * (option["zRatio_HR"]).  has_mask_ref: a reference exclusion mask will be
 * passed (its spline coefficients need room); has_phase_init: an initial
 * phase will be passed.  With the wrong-region correction (wr->enable) the
 * workspace also holds its buffers: a few bytes per voxel of each grid, and,
 * when a slice has more control points than the detection's shared-memory
 * working set holds (about 6000), 8 B times the next power of two above
 * the slice's control-point count plus 24 B per control point, for every
 * slice.
 */
WR_API int wr_xres_workspace_size(int32_t nz, int32_t ny, int32_t nx, int32_t nzh, int32_t nyh, int32_t nxh,
                                  const WrLKParams* p, float zRatio_HR, int32_t has_mask_ref, int32_t has_phase_init,
                                  const WrXresWrongRegion* wr, size_t* bytes);

/*
 * getMotion_v2; wr NULL or wr->enable = 0 runs it without the wrong-region
 * correction (option["wrong_region_enable"] = False).  The correction needs
 * p->iter >= 2 to change anything (with one iteration no pass updates the
 * motion).
 *   mov            (nz, ny, nx) float32 moving stack
 *   ref            (nzh, nyh, nxh) float32 reference stack
 *   excl_mask_mov  (nz, ny, nx) uint8 or NULL; excl_mask_ref (nzh, nyh, nxh)
 *                  uint8 or NULL: option["mask_mov"] / ["mask_ref"], values
 *                  resized per level and excluded where > 0.5
 *   motion_init    (nz, ny, nx, 3) or NULL: option["motion"]
 *   phase_init     (nz, ny, nx, 3) or NULL: option["phase"], the moving grid's
 *                  map into the reference (per level resized and divided by
 *                  the level's scale, :1978-1992); NULL: (x, y, z zRatio / zRatio_HR)
 *   p              layer, iter, r, zRatio, smoothPenalty, movRange, tol,
 *                  forced_updates (replay, -1 = off), flags (launch shape)
 * Outputs (any may be NULL): phase_out and motion_out (nz, ny, nx, 3),
 * ref_sampled_out (nz, ny, nx) = the reference's spline at the phase;
 * stats as for wr_lk_register (device or host-pinned WrLKStats).
 */
WR_API int wr_xres_register(const float* mov, int32_t nz, int32_t ny, int32_t nx, const float* ref, int32_t nzh,
                            int32_t nyh, int32_t nxh, const uint8_t* excl_mask_mov, const uint8_t* excl_mask_ref,
                            const float* motion_init, const float* phase_init, const WrLKParams* p,
                            float zRatio_HR, const WrXresWrongRegion* wr, float* phase_out,
                            float* motion_out, float* ref_sampled_out, WrLKStats* stats, void* workspace,
                            size_t workspace_bytes, void* stream);

/*
 * The continuous reference H (utils/calFlowCrossResolution.py:463-478,
 * 1144-1154): cubic B-spline of vol (nz, ny, nx) float32, map_coordinates
 * order 3, mode "nearest", at n points coords (n, 3) = (x, y, z) in vol's
 * index space; out (n) float32.  Workspace from wr_spline_workspace_size.
 */
WR_API int wr_spline_workspace_size(int32_t nz, int32_t ny, int32_t nx, size_t* bytes);
WR_API int wr_spline_sample(const float* vol, int32_t nz, int32_t ny, int32_t nx, const float* coords, int64_t n,
                            float* out, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Fixed-plane projections of mapped samples (utils/calFlowCrossResolution.py:
 * 480-569 + 878-1141 and 571-660 + 700-876): n samples values (n) at
 * coords (n, 3) = (x, y, z) in reference space, nplanes target z values;
 * output planes (nplanes, xout, yout) float32 with xout = ceil(xref / ds),
 * yout = ceil(yref / ds) (the reference's internal "zxy" order).
 *
 * wr_project_planes_max: max of the samples within z_window of a plane over
 * the XY pixels a sample reaches (nearest != 0: the rounded pixel; else
 * floor .. floor + 1, widened by extra_radius); values are shifted by
 * max(1 - min, 0) for the max and back, as the reference does; pixels
 * without a sample get fill_value (has_fill) or -inf.
 *
 * wr_project_planes_weighted: bilinear XY splat of the samples with z weight
 * mode 0 hard, 1 triangular, 2 gaussian (z_sigma <= 0: z_window / 2);
 * out = sum(v w) / sum(w) where sum(w) > eps, else fill_value; weight_out
 * (may be NULL) receives sum(w).
 *
 * Workspace: 8 bytes per output pixel plus 256 (wr_project_workspace_size).
 */
WR_API int wr_project_workspace_size(int32_t nplanes, int32_t xref, int32_t yref, int32_t ds, size_t* bytes);
WR_API int wr_project_planes_max(const float* values, const float* coords, int64_t n, const float* target_z,
                                 int32_t nplanes, int32_t xref, int32_t yref, int32_t ds, float z_window,
                                 int32_t nearest, int32_t extra_radius, float fill_value, int32_t has_fill, float* out,
                                 void* workspace, size_t workspace_bytes, void* stream);
WR_API int wr_project_planes_weighted(const float* values, const float* coords, int64_t n, const float* target_z,
                                      int32_t nplanes, int32_t xref, int32_t yref, int32_t ds, float z_window,
                                      float z_sigma, int32_t mode, float fill_value, float eps, float* out,
                                      float* weight_out, void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WR_XRES_H */
