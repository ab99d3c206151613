// Host-side plan of one registration call: level geometry, workspace layout
// and the device-resident control state.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include "wr_b200.h"

namespace wr {

// Field sources of a level's first iteration.
enum FieldMode { FIELD_CP = 0, FIELD_UP = 1, FIELD_DENSE = 2, FIELD_ZERO = 3 };

// Shift-invariant interior of a resize table: for outputs lo <= o < hi the
// taps read in[s * o + c0 + t], t < P, with the same weights w[t] for every
// such output (integer down-scale factor s).  hi <= lo: no such interior.
constexpr int kSIMaxTaps = 40;
// A row staged in shared memory in polyphase order (element e at
// (e mod s) * ls + e / s) gives tap t of output o at off[t] + o: the lanes of
// a warp, holding consecutive outputs, then read consecutive words.
struct SITaps {
  int P, s, c0, lo, hi;
  int ls;                 // polyphase row length, in_len / s + 1
  double w[kSIMaxTaps];
  float wf[kSIMaxTaps];   // the same weights rounded to float32
  int off[kSIMaxTaps];
  double wsum;            // the weights summed in tap order in float64
};

struct LevelPlan {
  int nx, ny, nz;     // level extent (x fastest)
  int ncx, ncy;       // control points per slice along x and y
  int ntx, nty;       // tiles: one per window plus a leftover tile if needed
  long long n;        // voxels
  long long ncp;      // control points (ncx * ncy * nz)
  long long nblk;     // CTAs of the fused iteration kernel
  float zratio;       // zRatio / 2^layer
  double zratio_d;
  // pass order of the separable resize from full resolution (x first when
  // the x scale is not larger than the y scale, like a stable argsort)
  int x_first;
  int up_x_first;
  int tx_taps, ty_taps;   // candidate taps of the full-res -> level tables
  SITaps six, siy;        // their shift-invariant interiors
  // workspace byte offsets
  size_t ref, movg, mbits, mmov, cp, sums, dense, errpart, penpart;
  size_t tx_w, tx_i, ty_w, ty_i;      // bicubic tables full-res -> level (float64)
  size_t ux_w, ux_i, uy_w, uy_i;      // bilinear tables level+1 -> level (2 taps, float)
};

struct Plan {
  int nz, ny, nx;
  int levels;          // layer + 1, index = layer
  int r, w, iter;
  bool has_mref, has_mmov, has_init, dense_all;
  // dense_out[l]: level l makes no update (iter == 1, or a replay of zero
  // updates), so its field stays the dense initial field; dense_in[l]: level l
  // starts from a dense field in its own buffer (it is dense_out, or the
  // coarser level is, whose dense field the up-sampling must read)
  bool dense_out[WR_MAX_LEVELS], dense_in[WR_MAX_LEVELS];
  int precision;
  LevelPlan lv[WR_MAX_LEVELS];
  size_t tmp_a, tmp_a_bytes, tmp_b, tmp_b_bytes;
  size_t tab_scratch;  // row-major x tables before their transpose
  size_t state;
  size_t total;
};

// Device control state of one call (lives in the workspace).
struct LKState {
  int active;          // the current level is still iterating
  int do_update;       // the last error evaluation asked for a motion update
  int level;
  int n_updates;       // updates done at the current level
  unsigned maxdiff_bits;
  int flags;
  double old_err[3];
  WrLKStats stats;
};

// Fills `plan` for a (nz, ny, nx) volume; returns WR_OK or an argument error.
int make_plan(int nz, int ny, int nx, const WrLKParams* p, bool has_mref, bool has_mmov,
              bool has_init, Plan* plan, const char** why);

}  // namespace wr
