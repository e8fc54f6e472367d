// tiles.cuh — records shared by the batched tile path of the terrain
// correction (tc.cu) and the batched speckle/crop stage (speckle.cu).
#pragma once

#include "runtime.cuh"

namespace sd {

constexpr int SP_MAX_HALF = 7;  // largest half window a tile batch may filter with (15 x 15)

// One tile of the speckle/crop stage: the tile's geocoded raster was computed
// on the tile grid widened by `halo` pixels on every side.
struct SpJob {
  const float *in;  // (rows + 2 halo) x (cols + 2 halo)
  const float *cos_in;
  const uint8_t *mask_in;
  float *out;  // rows x cols
  float *cos_out;
  uint8_t *mask_out;
  int64_t rows, cols;
  int halo;
  int kind;  // SD_SPECKLE_*, or -1: crop only
  int half;
  float enl, damping, cv_n_sq, cv_max_sq;
  int pad;
};

struct SpWork {
  int n_jobs;
  int tx, ty;  // block shape (= blockDim) the item prefix was computed for
  int pad;
  const SpJob *jobs;
  const uint64_t *pre;  // n_jobs + 1: exclusive prefix of tx x ty blocks
};

// k_main in its parameter form for one terrain-correction job record (the
// TcDev layout of tc_kernels.cuh), on stream st.
int launch_main_param(sd_ctx *ctx, const void *job, cudaStream_t st);
int speckle_validate(uint64_t len, uint64_t cols, uint64_t rows, int kind, uint64_t window, float enl,
                     float damping);
void speckle_coefs(int kind, uint64_t window, float enl, float damping, SpJob *j);
uint64_t speckle_tile_items(const SpJob &j, int tx, int ty);
int speckle_tiles_launch(sd_ctx *ctx, const SpWork *d_work, uint64_t total, bool full_grid, int tx, int ty);
bool speckle_shape_ok(int tx, int ty);

}  // namespace sd
