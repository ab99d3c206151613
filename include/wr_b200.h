/*
 * wr_b200.h - C ABI of the B200-native pyramid Lucas-Kanade registration path.
 *
 * The functions below replace, one for one, the reference package's
 * registration entry points (paths relative to src/wholistic_registration/):
 *
 *   wr_lk_register       utils/calFlow3d_Wei_v1.py:295-673   getMotion(dat_mov, dat_ref, option)
 *   wr_warp_trilinear    utils/calFlow3d_Wei_v1.py:676-706   correctMotion(data_raw, motion_field)
 *   wr_penalty_factor    utils/preprocess.py:42-66           getSmPnltNormFctr(dat_ref, option)
 *   wr_resize_table      utils/imresize.py:60-82             contributions(...) (host, no GPU needed)
 *
 * Conventions
 *   - Volumes are C-contiguous (z, y, x): x is the fastest axis.  The reference
 *     indexes the same memory as (x, y, z) after its (2, 1, 0) transpose
 *     (utils/registration.py:251,313), so "axis 0" there is x here.
 *   - Motion fields are (z, y, x, 3) float32 with [...,0] = dx, [...,1] = dy,
 *     [...,2] = dz: component c displaces axis c, exactly the reference's
 *     field transposed by (2, 1, 0, 3) (utils/registration.py:346).
 *   - Exclusion masks are (z, y, x) uint8, nonzero = excluded (outlier), the
 *     polarity of option["mask_ref"] / option["mask_mov"].  NULL = nothing
 *     excluded.
 *   - All data pointers are device pointers owned by the caller; work buffers
 *     come from the caller too (see wr_lk_workspace_size).  No entry point
 *     allocates or keeps global state, so calls on different streams with
 *     different workspaces may run concurrently.
 *   - Return codes: 0 = ok, > 0 = invalid argument (WR_E_*), < 0 = CUDA
 *     error (negated cudaError_t).  A message for the last failure on the
 *     calling thread is available from wr_last_error().
 */
#ifndef WR_B200_H
#define WR_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define WR_API __attribute__((visibility("default")))
#else
#define WR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define WR_ABI_VERSION 1
#define WR_MAX_LEVELS 8
#define WR_MAX_ITERS 64
#define WR_MAX_BATCH 64

/* element types of input volumes */
enum {
  WR_U8 = 1,
  WR_U16 = 2,
  WR_F32 = 3
};

/* argument errors */
enum {
  WR_OK = 0,
  WR_E_NULL = 1,        /* a required pointer is NULL */
  WR_E_SHAPE = 2,       /* shapes disagree or are out of range */
  WR_E_PARAM = 3,       /* a parameter is out of range */
  WR_E_DTYPE = 4,       /* unsupported element type */
  WR_E_WORKSPACE = 5,   /* workspace too small or misaligned */
  WR_E_NOCP = 6         /* some pyramid level has no control point */
};

/* storage precision of pyramid levels inside the solver */
enum {
  WR_PREC_F32 = 0,   /* plain path: levels, gradients and warps in float32 */
  WR_PREC_F16 = 1,   /* mixed: levels and gradients stored as float16 */
  WR_PREC_BF16 = 2   /* mixed: levels and gradients stored as bfloat16 */
};

/* WrLKParams.flags */
enum {
  /* The workspace already holds the pyramid of this `ref` and `excl_mask_ref`
     from an earlier call with the same shape and parameters: skip rebuilding
     them (a time series registered against one template). */
  WR_LK_REUSE_REFERENCE = 1,
  /* Tuning of the fused iteration kernel (results do not depend on it):
     visit the (z, window) tiles x-fastest instead of z-fastest ... */
  WR_LK_TILE_ORDER_X = 1 << 8,
  /* ... and run WR_LK_CTAS_PER_SM(n) persistent CTAs per SM, n in 1..15
     (0 = as many as fit). */
  WR_LK_CTAS_PER_SM_SHIFT = 12,
  WR_LK_CTAS_PER_SM_MASK = 15 << 12
};
#define WR_LK_CTAS_PER_SM(n) (((n) & 15) << WR_LK_CTAS_PER_SM_SHIFT)

/* A volume: device pointer, element type and (z, y, x) extent. */
typedef struct {
  const void* data;
  int32_t dtype;
  int32_t nz, ny, nx;
} WrVolume;

/*
 * Solver parameters: the keys getMotion reads from its option dict
 * (utils/calFlow3d_Wei_v1.py:318-324,429-431; defaults in utils/__init__.py:79-95).
 */
typedef struct {
  int32_t layer;          /* option["layer"]: levels = layer + 1 */
  int32_t iter;           /* option["iter"]: max error evaluations per level */
  int32_t r;              /* option["r"]: patch (2r+1) x (2r+1) x 1, CP stride 2r+1 */
  float zRatio;           /* option["zRatio"] at full resolution */
  float movRange;         /* option["movRange"]: max CP update length */
  double smoothPenalty;   /* option["smoothPenalty"], already normalised */
  double tol;             /* option["tol"]: |delta error| stopping threshold */
  int32_t precision;      /* WR_PREC_* */
  int32_t flags;          /* WR_LK_* bits */
  /* -1: the reference's stopping rules; n >= 0: perform exactly n motion
     updates at that level (replays another run's iteration counts) */
  int32_t forced_updates[WR_MAX_LEVELS];
} WrLKParams;

/* Per-call statistics (device memory), the scalar part of getMotion's error_log. */
typedef struct {
  int32_t levels;                         /* layer + 1 */
  int32_t evals[WR_MAX_LEVELS];           /* error evaluations per level, index = layer */
  int32_t updates[WR_MAX_LEVELS];         /* motion updates per level */
  int32_t nan_solves;                     /* CP solve components that were NaN (set to 0) */
  int32_t fp64_solves;                    /* mixed precision: CP solves redone in float64 */
  double current_error;                   /* last evaluated error (returned by getMotion) */
  double diff_error[WR_MAX_LEVELS][WR_MAX_ITERS];
  double penalty_error[WR_MAX_LEVELS][WR_MAX_ITERS];
  double max_diff_motion[WR_MAX_LEVELS][WR_MAX_ITERS];
} WrLKStats;

/* ABI version of the loaded library (WR_ABI_VERSION). */
WR_API int wr_abi_version(void);

/* Message describing the last failed call on this thread ("" if none). */
WR_API const char* wr_last_error(void);

/*
 * Bytes of device workspace wr_lk_register needs for this volume shape and
 * parameters.  Host-only; needs no GPU.  Replaces the device arrays getMotion
 * allocates per level (utils/calFlow3d_Wei_v1.py:346-439).
 */
WR_API int wr_lk_workspace_size(int32_t nz, int32_t ny, int32_t nx, const WrLKParams* p,
                         size_t* bytes);

/*
 * Register `mov` onto `ref`: getMotion (utils/calFlow3d_Wei_v1.py:295-673).
 *   mov, ref       : same shape; WR_U8, WR_U16 or WR_F32 elements
 *   excl_mask_mov  : option["mask_mov"], (z,y,x) uint8 or NULL
 *   excl_mask_ref  : option["mask_ref"], (z,y,x) uint8 or NULL
 *   motion_init    : option["motion"], (z,y,x,3) float32 or NULL
 *   motion_out     : (z,y,x,3) float32 result
 *   stats          : device WrLKStats or NULL
 *   workspace      : >= wr_lk_workspace_size bytes, 256-byte aligned
 * Asynchronous on `stream` (a cudaStream_t; NULL = legacy default stream).
 */
WR_API int wr_lk_register(const WrVolume* mov, const WrVolume* ref, const uint8_t* excl_mask_mov,
                   const uint8_t* excl_mask_ref, const WrLKParams* p, const float* motion_init,
                   float* motion_out, WrLKStats* stats, void* workspace, size_t workspace_bytes,
                   void* stream);

/*
 * Instrumentation of one wr_lk_register_profiled call.  The caller creates
 * timing-enabled CUDA events; the library records acc_begin[i] / acc_end[i]
 * on the call's stream around the i-th launch of the fused iteration kernel
 * (the dominant kernel), in launch order: levels from coarsest to finest,
 * `iter` launches per level.  `launches` returns the number of kernels the
 * call put on the stream.
 */
typedef struct {
  void* const* acc_begin;   /* cudaEvent_t[capacity] */
  void* const* acc_end;     /* cudaEvent_t[capacity] */
  int32_t capacity;
  int32_t recorded;         /* out: event pairs recorded */
  int32_t launches;         /* out: kernels launched */
  int32_t pad;
} WrProfile;

/* wr_lk_register with instrumentation (prof may be NULL). No reference counterpart:
   it exists to time the fused iteration kernel inside a full registration. */
WR_API int wr_lk_register_profiled(const WrVolume* mov, const WrVolume* ref, const uint8_t* excl_mask_mov,
                                   const uint8_t* excl_mask_ref, const WrLKParams* p, const float* motion_init,
                                   float* motion_out, WrLKStats* stats, void* workspace, size_t workspace_bytes,
                                   void* stream, WrProfile* prof);

/*
 * Snapshots getMotion keeps in its error_log (utils/calFlow3d_Wei_v1.py:
 * 329-353, 451-470): at every iteration `it` of level l with
 * it % save_ite == 0, taken before that iteration's update, the level's dense
 * motion ("motion_current") and the moving level warped by it
 * ("data_mov_corrected", trilinear with edge clamping); once per level the
 * level's reference and moving images ("data_ref", "data_mov").  All device
 * float32 (z, y_l, x_l[, 3]) arrays, x_l / y_l the level's extents; slot s of
 * level l holds iteration s * save_ite (capacity slots per level; the level
 * evaluated stats.evals[l] times, so ceil(evals / save_ite) slots are
 * written, at most capacity).  Any pointer may be NULL.
 */
typedef struct {
  int32_t save_ite;
  int32_t capacity;
  float* motion[WR_MAX_LEVELS];
  float* warped[WR_MAX_LEVELS];
  float* level_ref[WR_MAX_LEVELS];
  float* level_mov[WR_MAX_LEVELS];
} WrSnapshots;

/* wr_lk_register that also fills `snap` (getMotion's error_log snapshots);
   snap may be NULL. */
WR_API int wr_lk_register_snapshots(const WrVolume* mov, const WrVolume* ref, const uint8_t* excl_mask_mov,
                                    const uint8_t* excl_mask_ref, const WrLKParams* p, const float* motion_init,
                                    float* motion_out, WrLKStats* stats, void* workspace, size_t workspace_bytes,
                                    void* stream, const WrSnapshots* snap);

/*
 * One frame of a batched registration (wr_lk_register_batch).  mov and ref
 * have the same shape and dtype; shapes may differ between frames.
 */
typedef struct {
  WrVolume mov;
  WrVolume ref;
  const uint8_t* excl_mask_mov;   /* or NULL */
  const uint8_t* excl_mask_ref;   /* or NULL */
  const float* motion_init;       /* option["motion"] or NULL */
  float* motion_out;              /* (z,y,x,3) float32 */
  float* warped_out;              /* correctMotion(mov, motion) (z,y,x) float32, or NULL */
  WrLKStats* stats;               /* device WrLKStats or NULL */
} WrLKItem;

/* Workspace bytes of wr_lk_register_batch for these frames and parameters
   (only the shapes, dtypes and the presence of masks / initial fields are
   read). */
WR_API int wr_lk_batch_workspace_size(const WrLKItem* items, int32_t n, const WrLKParams* p, size_t* bytes);

/*
 * getMotion (and optionally correctMotion) of n <= WR_MAX_BATCH frames with
 * one parameter set, as the reference's batch loop calls it frame by frame
 * (utils/registration.py:299-346), but run together: each pyramid level
 * advances every frame with one persistent launch of the fused iteration
 * kernel per LK iteration (plus one launch each of the decision, solve and
 * bookkeeping kernels), each frame keeping its own stopping state, so every
 * frame's results equal those of a wr_lk_register call on it alone.
 * The frames must agree on dtype and on which of the masks and motion_init
 * are present.  WR_LK_REUSE_REFERENCE keeps each frame's reference pyramid
 * from the previous batch call on the same workspace.  No profiling.
 */
WR_API int wr_lk_register_batch(const WrLKItem* items, int32_t n, const WrLKParams* p, void* workspace,
                                size_t workspace_bytes, void* stream);

/*
 * wr_lk_register_batch with one parameter set per frame (params[i] for
 * items[i]), the reference's batch loop (utils/registration.py:299-346) run
 * over volumes that each carry their own option dict: patch radius r, layer,
 * iter, zRatio, movRange, smoothPenalty, tol and forced_updates may differ
 * between frames; precision and the launch-shape flags (WR_LK_TILE_ORDER_X,
 * WR_LK_CTAS_PER_SM_*) must agree.  Level l (0 = finest) of every frame that
 * has it runs together, one persistent launch of the fused iteration kernel
 * per LK iteration and field kind; each frame's results equal those of a
 * wr_lk_register call on it with its own parameters.
 */
WR_API int wr_lk_batch_each_workspace_size(const WrLKItem* items, const WrLKParams* params, int32_t n,
                                           size_t* bytes);
WR_API int wr_lk_register_batch_each(const WrLKItem* items, const WrLKParams* params, int32_t n, void* workspace,
                                     size_t workspace_bytes, void* stream);

/*
 * getMotion followed by correctMotion of the same moving volume, the step the
 * reference's series registration takes per frame
 * (motion = getMotion(mov, ref, option); out = correctMotion(mov, motion)):
 * replaces a wr_lk_register + wr_warp_trilinear(mov) pair with the same
 * results, writing motion_out and warped_out ((z,y,x) float32) in one pass
 * over the full-resolution grid.  prof may be NULL.  No single reference
 * function corresponds to it.
 */
WR_API int wr_lk_register_warp(const WrVolume* mov, const WrVolume* ref, const uint8_t* excl_mask_mov,
                               const uint8_t* excl_mask_ref, const WrLKParams* p, const float* motion_init,
                               float* motion_out, float* warped_out, WrLKStats* stats, void* workspace,
                               size_t workspace_bytes, void* stream, WrProfile* prof);

/*
 * Pull-warp `src` through `motion`: out(p) = src(p + motion(p)), trilinear,
 * edge-replicated, float32 result (correctMotion, utils/calFlow3d_Wei_v1.py:676-706).
 *   motion : (z,y,x,3) float32 device; out : (z,y,x) float32 device.
 */
WR_API int wr_warp_trilinear(const WrVolume* src, const float* motion, float* out, void* stream);

/*
 * Smoothness-penalty normalisation factor of `ref` over voxels not excluded by
 * excl_mask_ref (getSmPnltNormFctr, utils/preprocess.py:42-66).  Writes one
 * double to the device pointer `factor_out`.
 */
WR_API int wr_penalty_factor(const WrVolume* ref, const uint8_t* excl_mask_ref, double* factor_out,
                      void* scratch, size_t scratch_bytes, void* stream);

/*
 * wr_penalty_factor for callers that cannot allocate device memory: no
 * counterpart in the reference (whose NumPy/CuPy code allocates freely).
 * Callers that embed the library in a host application whose device memory
 * is owned by its own pool (a stray cudaMalloc would fail or break the pool's
 * accounting), or acquisition loops that must not enter the allocator
 * between frames, call this form: it takes the same inputs and output as
 * wr_penalty_factor and allocates nothing.  Its per-block partial sums live
 * in a 256 KiB static device array that every device loading the library
 * holds until exit; volumes above 134,217,728 voxels (128 x 1024 x 1024) are
 * rejected with WR_E_SHAPE.  The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current, so
 * make that first call before any stream capture.  All calls share the
 * array: calls that overlap on the GPU (other streams, other threads) race
 * and must be serialised by the caller.  Nothing in the array needs to start
 * at zero; each call writes every slot it reads.
 */
WR_API int wr_penalty_factor_noalloc(const WrVolume* ref, const uint8_t* excl_mask_ref, double* factor_out,
                                     void* stream);

/* Scratch bytes wr_penalty_factor needs for this shape. */
WR_API int wr_penalty_factor_scratch(int32_t nz, int32_t ny, int32_t nx, size_t* bytes);

/*
 * Resize tap table along one axis, host-side (contributions,
 * utils/imresize.py:60-82), before zero-column removal: for each of `out_len`
 * outputs, `*taps` candidate taps (weights float64 and source indices).
 * method 0 = bicubic (antialiased when shrinking), 1 = bilinear.
 * Call with weights == NULL to get `*taps`.
 */
WR_API int wr_resize_table(int32_t in_len, int32_t out_len, int32_t method, double* weights,
                    int32_t* indices, int32_t* taps);

#ifdef __cplusplus
}
#endif

#endif /* WR_B200_H */
