/*
 * Outlier masks of the per-batch registration wrapper on the device.
 *
 *   wr_get_mask     <- getMask(dat, thresFactor)          utils/mask.py:59-111
 *                      (robust_mean_std, utils/preprocess.py:69-84)
 *   wr_bwareafilt3  <- bwareafilt3_wei(mask, maskRange)    utils/mask.py:8-56
 *
 * Volumes are (z, y, x) C-contiguous device arrays (the reference's (x, y, z)
 * arrays are the same memory).  Return codes as in wr_b200.h; the last error
 * message of the calling thread is wr_mask_last_error().  Asynchronous on
 * `stream`.
 */
#ifndef WR_MASK_H
#define WR_MASK_H

#include <stddef.h>
#include <stdint.h>

#include "wr_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

WR_API const char* wr_mask_last_error(void);

/* Workspace bytes of wr_get_mask and wr_bwareafilt3 for a volume. */
WR_API int wr_mask_workspace_size(int32_t nz, int32_t ny, int32_t nx, size_t* bytes);

/*
 * getMask: mu, sigma = mean and standard deviation of the values at or below
 * the `percentile`-th percentile (numpy's "linear" percentile of the float32
 * data, from exact order statistics found by radix selection); mask =
 * |(v - mu) / sigma| > thres_factor in float32; then a 3x3 (per z slice)
 * binary opening and a 3x3 binary dilation (scikit-image semantics: erosion
 * treats the outside as set, dilation as clear).  mu and sigma are summed in
 * float64 in a fixed order and rounded to float32 (numpy sums float32
 * pairwise), so a voxel whose z-score lies within a few float32 ulps of
 * thres_factor may classify differently.  stats_out (device, optional)
 * receives mu, sigma and the percentile value as three doubles.  The
 * reference calls it with percentile 95.
 */
WR_API int wr_get_mask(const WrVolume* vol, double thres_factor, double percentile, uint8_t* mask_out,
                       double* stats_out, void* workspace, size_t workspace_bytes, void* stream);

/*
 * bwareafilt3_wei: keep the 26-connected components of mask_in (nonzero =
 * set) whose voxel count lies in [min_size, max_size]; mask_out is 0/1.
 * n_components (device, optional) receives the number of components kept;
 * error_flag (device, optional) is nonzero if a union-find retry loop hit its
 * bound (it does not on any input; the flag makes the bound observable).
 */
/*
 * Frame correlation of pick_initial_reference (utils/reference.py:60-78):
 * `frames` is t rows of d float32 values (device); writes each row's mean
 * (`means`, t doubles) and the Gram matrix of the demeaned rows (`gram`,
 * t x t doubles, symmetric), both summed in float64 in a fixed order.  The
 * caller normalises it by the square roots of its diagonal as the reference
 * does.  1 <= t <= 4096.
 */
WR_API int wr_frame_gram(const float* frames, int32_t t, int64_t d, double* means, double* gram, void* stream);

WR_API int wr_bwareafilt3(const uint8_t* mask_in, int32_t nz, int32_t ny, int32_t nx, int64_t min_size,
                          int64_t max_size, uint8_t* mask_out, int32_t* n_components, int32_t* error_flag,
                          void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WR_MASK_H */
