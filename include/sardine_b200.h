/*
 * sardine_b200.h — C ABI of the B200 (sm_100a) implementation of SARdine's
 * data-parallel hot path: sigma0 LUT calibration with NESZ, TOPS midpoint
 * deburst, IW merge, backward Range-Doppler terrain correction and the
 * SpeckleKernel filters.
 *
 * Conventions
 *  - Every entry point returns an int status (sd_status).  Status codes map
 *    one-to-one onto the Rust error variants of the function each entry point
 *    replaces; sd_last_error() returns the formatted message of the last
 *    failure on a context.  Nothing here aborts the process.
 *  - Times are int64 microseconds since an arbitrary common epoch.  The
 *    reference keeps chrono DateTime values but only ever uses whole-
 *    microsecond differences of them (Duration::num_microseconds), so this is
 *    lossless for annotation times (which carry microseconds).
 *  - Array pointers may be host memory (pageable or pinned) or device memory
 *    of the context's device; the library detects which and stages host
 *    buffers itself.  With device pointers the call enqueues on the
 *    context's stream and returns after the stream has finished, unless the
 *    entry point says otherwise.
 *  - A context is not thread-safe: use one context per host thread.
 *
 * Reference paths cited as file:line are relative to the SARdine repository
 * (sardine/src/...).
 */
#ifndef SARDINE_B200_H
#define SARDINE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SD_ABI_VERSION 1

/* ── Status codes ─────────────────────────────────────────────────────── */
typedef enum sd_status {
    SD_OK = 0,
    SD_ERR_INVALID_ARGUMENT = 1,
    SD_ERR_CUDA = 2,
    SD_ERR_OUT_OF_MEMORY = 3,
    SD_ERR_INTERNAL = 4,
    SD_ERR_TIMEOUT = 5,
    SD_ERR_BUSY = 6,
    /* TerrainCorrectionError (terrain_correction.rs:45-67) */
    SD_ERR_TC_ORBIT = 10,          /* OrbitError::OutsideOrbitWindow / InsufficientCoverage */
    SD_ERR_TC_DEM = 11,
    SD_ERR_TC_NO_GRID_POINTS = 12,
    SD_ERR_TC_NO_SUBSWATHS = 13,
    SD_ERR_TC_CONFIG = 14,
    SD_ERR_TC_PROJECTION = 15,
    /* SpeckleError (speckle.rs:96-108) */
    SD_ERR_SPECKLE_DIMENSION_MISMATCH = 20,
    SD_ERR_SPECKLE_BAD_WINDOW = 21,
    SD_ERR_SPECKLE_BAD_ENL = 22,
    SD_ERR_SPECKLE_BAD_DAMPING = 23,
    /* CalibrationError (apply_calibration.rs:64-84) */
    SD_ERR_CAL_NO_CALIBRATION_VECTORS = 30,
    SD_ERR_CAL_NO_NOISE_RANGE_VECTORS = 31,
    SD_ERR_CAL_LUT_RANGE_INSUFFICIENT = 32,
    /* DeburstError (deburst.rs:56-121) */
    SD_ERR_DEBURST_NO_BURSTS = 40,
    SD_ERR_DEBURST_BURST_COUNT_MISMATCH = 41,
    SD_ERR_DEBURST_TIFF_TOO_SMALL = 42,
    SD_ERR_DEBURST_EMPTY_VALID_WINDOW = 43,
    SD_ERR_DEBURST_INVALID_OVERLAP = 44,
    SD_ERR_DEBURST_IMPLAUSIBLE_OVERLAP = 45,
    /* MergeError (merge_subswaths.rs:62-81) */
    SD_ERR_MERGE_EMPTY_INPUTS = 50,
    SD_ERR_MERGE_INCONSISTENT_PIXEL_SPACING = 51,
    SD_ERR_MERGE_EMPTY_SWATH = 52,
    /* ExportError (export.rs:25-40) */
    SD_ERR_EXPORT_IO = 60,
    SD_ERR_EXPORT_INVALID_NOISE_FLOOR = 61,
    SD_ERR_EXPORT_INVALID_GEOTRANSFORM = 62,
    SD_ERR_EXPORT_INVALID_TILE_SIZE = 63,
    /* SlcReadError (slc_reader.rs:66-98; the multi-slice variants are out of scope) */
    SD_ERR_SLC_IO = 70,
    SD_ERR_SLC_NOT_TIFF = 71,
    SD_ERR_SLC_BIGTIFF = 72,
    SD_ERR_SLC_MISSING_TAG = 73,
    SD_ERR_SLC_UNSUPPORTED_FORMAT = 74,
    SD_ERR_SLC_NON_CONTIGUOUS_STRIPS = 75,
    SD_ERR_SLC_LINE_OUT_OF_BOUNDS = 76,
    /* GroundRangeError (ground_range.rs:42-57) */
    SD_ERR_GRD_NO_GRID_POINTS = 80,
    SD_ERR_GRD_EMPTY_IMAGE = 81,
    SD_ERR_GRD_INVALID_SPACING = 82,
    SD_ERR_GRD_INVALID_AZIMUTH_SPACING = 83,
    SD_ERR_GRD_INTERPOLATION_FAILED = 84,
    /* InsarError (insar/error.rs:7-33) */
    SD_ERR_INSAR_NO_DC_ESTIMATES = 90,
    SD_ERR_INSAR_AZIMUTH_TIME_BEFORE_DC = 91,
    SD_ERR_INSAR_INVALID_WINDOW_SIZE = 92,
    SD_ERR_INSAR_ORBIT = 93,
    SD_ERR_INSAR_COREG_GRID_TOO_SMALL = 94
} sd_status;

/* ── Enumerations mirroring the reference's enums ─────────────────────── */
/* ResamplingKernel (pipeline_options.rs:75-90) */
enum { SD_RESAMPLE_BILINEAR = 0, SD_RESAMPLE_BICUBIC = 1, SD_RESAMPLE_LANCZOS3 = 2 };
/* OutputCrs (output_crs.rs:70-96); LAEA and WebMercator are not supported */
enum { SD_CRS_WGS84 = 0, SD_CRS_UTM_NORTH = 1, SD_CRS_UTM_SOUTH = 2 };
/* DemSource implementations understood by the device path */
enum {
    SD_DEM_GEOGRAPHIC = 0,   /* one Glo30-style tile: dem.rs:351-371 semantics */
    SD_DEM_PROJECTED_UTM = 1 /* projected grid: forward UTM, then the same grid semantics */
};
/* GeoidModel (geoid.rs:342-402): Zero, or a 73x144 2.5-degree undulation grid */
enum { SD_GEOID_ZERO = 0, SD_GEOID_GRID = 1 };
/* SpeckleFilter (speckle.rs:61-91) */
enum {
    SD_SPECKLE_BOXCAR = 0, SD_SPECKLE_LEE = 1, SD_SPECKLE_FROST = 2,
    SD_SPECKLE_GAMMA_MAP = 3, SD_SPECKLE_REFINED_LEE = 4
};
/* Terrain-correction precision mode */
enum {
    SD_PRECISION_FP64 = 0,  /* reproduces the reference arithmetic (default) */
    SD_PRECISION_SPLIT = 1  /* FP64 orbit/anchor + FP32 bulk, error reported */
};
/* mask_code (terrain_correction.rs:346-376) */
enum {
    SD_MASK_VALID = 0, SD_MASK_OUTSIDE_FOOTPRINT = 1, SD_MASK_DEM_MISSING = 2,
    SD_MASK_NON_CONVERGED = 3, SD_MASK_DEGENERATE_GEOMETRY = 4, SD_MASK_SHADOW = 5,
    SD_MASK_LAYOVER = 6, SD_MASK_FORESHORTENING = 7, SD_MASK_NOISE_MASKED = 8,
    SD_MASK_DEM_NEIGHBOUR_MISSING = 9
};
#define SD_NEWTON_ITER_HIST_SIZE 16  /* NEWTON_ITER_HIST_SIZE, terrain_correction.rs:96 */

/* ── Data contracts ───────────────────────────────────────────────────── */

/* StateVector (types.rs:142); time as int64 us. */
typedef struct sd_state_vector {
    int64_t time_us;
    double position_m[3];
    double velocity_m_s[3];
} sd_state_vector;

/* RadarImage (pipeline_options.rs:100-135) as implemented by MergedSigma0
 * (terrain_correction.rs:888-928; merge_subswaths.rs:106-162). */
typedef struct sd_radar_image {
    const float *data;   /* lines x samples, row-major, NaN = nodata */
    const float *nesz;   /* same shape, or NULL (nesz_at -> None)    */
    uint64_t lines;
    uint64_t samples;
    int64_t azimuth_start_time_us;
    double near_slant_range_time_s;
    double range_pixel_spacing_m;
} sd_radar_image;

/* The parts of SceneMetadata (types.rs:406) the terrain correction reads. */
typedef struct sd_scene {
    double azimuth_time_interval_s;  /* scene.sub_swaths[0].azimuth_time_interval_s */
    int32_t n_sub_swaths;            /* 0 -> TerrainCorrectionError::NoSubSwaths */
    double min_lat_deg, max_lat_deg, min_lon_deg, max_lon_deg; /* bounding_box */
    const sd_state_vector *state_vectors; /* orbit.state_vectors, sorted by time */
    uint64_t n_state_vectors;
} sd_scene;

/* DemSource (dem.rs:829-842).  (origin_y, origin_x) is the centre of pixel
 * (0,0): latitude/longitude in degrees for SD_DEM_GEOGRAPHIC, northing/easting
 * in metres for SD_DEM_PROJECTED_UTM.  Row 0 is the northern edge. */
typedef struct sd_dem {
    int32_t kind;
    int32_t utm_zone;    /* SD_DEM_PROJECTED_UTM only */
    int32_t utm_south;   /* SD_DEM_PROJECTED_UTM only */
    int32_t _pad;
    const float *data;   /* height x width, row-major, NaN = void */
    uint64_t width;
    uint64_t height;
    double origin_y;
    double origin_x;
    double pixel_size;
} sd_dem;

/* GeoidModel (geoid.rs:342-402). */
typedef struct sd_geoid {
    int32_t kind;                 /* SD_GEOID_ZERO or SD_GEOID_GRID */
    int32_t _pad;
    const float *undulations_m;   /* 73 x 144, row 0 = 90N, col 0 = 0E */
} sd_geoid;

/* GeolocationGridPoint (types.rs:171): the two fields the terrain correction
 * uses to seed its azimuth-time guess (terrain_correction.rs:1080-1137).
 * Pass the points of IW2, or of the first sub-swath when IW2 is absent. */
typedef struct sd_geo_grid_point {
    int64_t azimuth_time_us;
    double latitude_deg;
} sd_geo_grid_point;

/* TerrainCorrectionConfig (terrain_correction.rs:100-236) plus the two
 * environment knobs the reference reads inside terrain_correction
 * (SARDINE_TC_PROJECTOR_ANCHORS, default 256; SARDINE_TC_ROW_CHUNK, which
 * only schedules CPU work and is accepted and ignored here). */
typedef struct sd_tc_config {
    double pixel_spacing;        /* pixel_spacing_deg, in CRS units */
    int32_t crs;                 /* SD_CRS_* */
    int32_t utm_zone;            /* 1..60 for UTM CRSs */
    int32_t max_newton_iterations;
    int32_t flatten;
    double newton_tolerance_s;
    int32_t compute_lia;
    int32_t resampling;          /* SD_RESAMPLE_* */
    float noise_floor_margin_db; /* -INFINITY disables NESZ masking */
    int32_t projector_anchors;   /* >= 1 */
    int32_t precision;           /* SD_PRECISION_* */
    int32_t _pad;
} sd_tc_config;

/* GeocodedImage (terrain_correction.rs:238-307) without the rasters. */
typedef struct sd_geocoded_info {
    uint64_t rows, cols;
    double origin_lat_deg, origin_lon_deg; /* top-left corner, CRS units */
    double pixel_spacing;
    double geotransform[6];
    uint64_t total_pixel_count;
    uint64_t valid_pixel_count;
    uint64_t dem_missing_count;
    uint64_t outside_footprint_count;
    uint64_t non_converged_count;
    uint64_t degenerate_geometry_count;
    uint64_t flat_masked_count;
    uint64_t noise_masked_count;
    uint64_t newton_iter_histogram[SD_NEWTON_ITER_HIST_SIZE];
    /* diagnostics (no reference counterpart): converged pixels whose
     * azimuth time fell outside the precomputed fixed-point pair, so their
     * outputs were computed on the row walk's exact path */
    uint64_t diag_exact_path_pixels;
    /* diagnostic (split precision): pixels whose FP32 outputs fell inside
     * their error margin and were recomputed in FP64 */
    uint64_t diag_fp64_redo_pixels;
    /* diagnostic (split precision): candidates whose FP32 resampling sum
     * cancelled beyond its error bound and was re-sampled in FP64 */
    uint64_t diag_fp64_resampled;
} sd_geocoded_info;

/* CalibrationVector / NoiseRangeVector (calibration.rs:38-82): one LUT row. */
typedef struct sd_lut_vector {
    int32_t line;
    int32_t _pad;
    const uint32_t *pixels;  /* ascending */
    const float *values;
    uint64_t n;
} sd_lut_vector;

/* NoiseAzimuthVector (calibration.rs:86-96); n == 0 means absent. */
typedef struct sd_noise_azimuth {
    const int32_t *lines;
    const float *values;
    uint64_t n;
} sd_noise_azimuth;

/* BurstEntry (types.rs:351). */
typedef struct sd_burst {
    int64_t azimuth_time_us;
    uint64_t burst_index;
    uint64_t first_line, last_line;
    uint64_t first_valid_sample, last_valid_sample;
} sd_burst;

/* The SubSwathMetadata (types.rs:281) fields deburst/merge read. */
typedef struct sd_subswath {
    uint64_t burst_count;
    uint64_t lines_per_burst;
    double azimuth_time_interval_s;
    double range_pixel_spacing_m;
    double slant_range_time_s;
} sd_subswath;

/* One IW sub-swath as fed to the fused calibrate+deburst+merge path:
 * the measurement raster (what SlcReader::read_burst_raw would return),
 * its metadata, bursts and LUTs. */
typedef struct sd_swath_input {
    const int16_t *slc_iq;        /* tiff_height x tiff_width x [I,Q] */
    uint64_t tiff_width, tiff_height;
    sd_subswath sw;
    const sd_burst *bursts;       /* sorted by burst_index */
    uint64_t n_bursts;
    const sd_lut_vector *cal;     /* sigmaNought vectors */
    uint64_t n_cal;
    const sd_lut_vector *noise_range;
    uint64_t n_noise_range;
    sd_noise_azimuth noise_azimuth;
} sd_swath_input;

/* MergedSigma0 metadata (merge_subswaths.rs:106-162). */
typedef struct sd_merged_info {
    uint64_t lines, samples;
    double near_slant_range_time_s;
    double range_pixel_spacing_s;
    double range_pixel_spacing_m;
    uint32_t cal_lut_extrapolation_gap_px;
    uint32_t noise_lut_extrapolation_gap_px;
    int64_t azimuth_start_time_us;
    /* per-swath layout, for diagnostics and the split/serving paths */
    int32_t n_swaths;
    int32_t _pad;
    int64_t swath_out_offset[8];
    uint64_t swath_seam[8];
    uint64_t swath_lines[8];
    uint64_t swath_valid_offset[8];
} sd_merged_info;

typedef struct sd_ctx sd_ctx;

/* ── Context ──────────────────────────────────────────────────────────── */
int sd_abi_version(void);
int sd_ctx_create(int device, sd_ctx **out);
void sd_ctx_destroy(sd_ctx *ctx);
const char *sd_last_error(const sd_ctx *ctx);
/* Number of this library's kernels launched on the context since creation. */
uint64_t sd_kernel_launches(const sd_ctx *ctx);
/* The context's CUDA stream (cudaStream_t), for callers that interleave work. */
void *sd_ctx_stream(sd_ctx *ctx);
/* Per-kernel timing: when on, every kernel launch is bracketed by CUDA events
 * on the context's stream and the durations accumulate per kernel name.
 * Turning it on clears the accumulators. */
int sd_ctx_set_timing(sd_ctx *ctx, int on);
/* Accumulated kernel times: names as a newline-separated list (same order as
 * ms/counts); *n_out = number of distinct kernels. */
int sd_ctx_kernel_times(sd_ctx *ctx, char *names, uint64_t names_len, double *ms,
                        uint64_t *counts, uint64_t max_entries, uint64_t *n_out);

/* ── Speckle ──────────────────────────────────────────────────────────────
 * Replaces SpeckleKernel::apply / apply_speckle_filter (speckle.rs:131-180,
 * 586-603).  window is ignored for SD_SPECKLE_REFINED_LEE (fixed 7x7);
 * enl is used by Lee, Gamma-MAP and Refined Lee, damping by Frost. */
int sd_speckle(sd_ctx *ctx, const float *data, uint64_t data_len, uint64_t cols,
               uint64_t rows, int32_t kind, uint64_t window, float enl,
               float damping, float *out);

/* ── Deburst ──────────────────────────────────────────────────────────────
 * compute_overlap_lines (deburst.rs:172-210). */
int sd_compute_overlap_lines(sd_ctx *ctx, const sd_burst *burst_k,
                             const sd_burst *burst_k1, double ati_s,
                             uint64_t lines_per_burst, uint64_t *overlap);
/* Output shape of deburst_subswath without running it. */
int sd_deburst_plan(sd_ctx *ctx, const sd_subswath *sw, const sd_burst *bursts,
                    uint64_t n_bursts, uint64_t tiff_height, uint64_t *lines,
                    uint64_t *samples, uint64_t *valid_sample_offset);
/* deburst_subswath (deburst.rs:230-344) over an in-memory measurement raster.
 * out_iq: lines x samples x [I,Q] int16. */
int sd_deburst_subswath(sd_ctx *ctx, const int16_t *slc_iq, uint64_t tiff_width,
                        uint64_t tiff_height, const sd_subswath *sw,
                        const sd_burst *bursts, uint64_t n_bursts, int16_t *out_iq);

/* ── Calibration ──────────────────────────────────────────────────────────
 * apply_calibration (apply_calibration.rs:374-572). */
int sd_apply_calibration(sd_ctx *ctx, const int16_t *deburst_iq, uint64_t lines,
                         uint64_t samples, uint64_t valid_sample_offset,
                         const sd_lut_vector *cal, uint64_t n_cal,
                         const sd_lut_vector *noise_range, uint64_t n_noise_range,
                         const sd_noise_azimuth *noise_azimuth,
                         uint64_t tiff_line_origin, float *out_sigma0,
                         float *out_nesz, uint32_t *cal_gap_px,
                         uint32_t *noise_gap_px);

/* Allocation-free variant of sd_apply_calibration — no counterpart in the
 * reference.  For callers that cannot allocate device memory while they run
 * (a process that reserved its HBM budget up front in its own pool, a stage
 * that must not let cudaMalloc/cudaFree serialise other streams, a host that
 * only lends this library buffers it already owns).  Same results as
 * sd_apply_calibration; no device allocation of any kind:
 *  - deburst_iq, out_sigma0 and out_nesz must be device (or managed) memory
 *    of the current device; the call is enqueued on `stream` (NULL = the
 *    legacy default stream) and returns without waiting for it;
 *  - working memory is one static 20 MiB device array inside the library,
 *    held by every device that loads it until the process exits.  Limits:
 *    <= 64 LUT vectors and <= 65536 LUT knots per family (sigma0, range
 *    noise), <= 32768 lines, <= 32768 samples; larger inputs are rejected
 *    with SD_ERR_INVALID_ARGUMENT and a message;
 *  - every call looks up the array's address on the current device
 *    (cudaGetSymbolAddress), and the first call on a device loads the
 *    library's module there: make that first call before any stream
 *    capture.  The call stages its LUT tables from host memory that lives
 *    only for the call, so it refuses a capturing stream
 *    (SD_ERR_INVALID_ARGUMENT);
 *  - a null LUT array with a non-zero count is rejected the same way;
 *  - every call shares the one array and leaves its contents behind (nothing
 *    in it needs to start at zero): calls whose work overlaps on the GPU race
 *    with each other, so serialise them (one stream, or events);
 *  - err (may be NULL) receives the error message, err_len bytes at most. */
int sd_apply_calibration_noalloc(void *stream, const int16_t *deburst_iq, uint64_t lines,
                                 uint64_t samples, uint64_t valid_sample_offset,
                                 const sd_lut_vector *cal, uint64_t n_cal,
                                 const sd_lut_vector *noise_range, uint64_t n_noise_range,
                                 const sd_noise_azimuth *noise_azimuth,
                                 uint64_t tiff_line_origin, float *out_sigma0,
                                 float *out_nesz, uint32_t *cal_gap_px,
                                 uint32_t *noise_gap_px, char *err, uint64_t err_len);

/* ── Merge ────────────────────────────────────────────────────────────────
 * merge_subswaths (merge_subswaths.rs:207-450) over n calibrated swaths,
 * given in IW1 < IW2 < IW3 order.  sigma0[i]/nesz[i] are lines[i] x
 * samples[i].  Call with out_data == NULL to only fill *info. */
int sd_merge_subswaths(sd_ctx *ctx, int32_t n, const float *const *sigma0,
                       const float *const *nesz, const uint64_t *lines,
                       const uint64_t *samples, const uint64_t *valid_sample_offset,
                       const uint32_t *cal_gap_px, const uint32_t *noise_gap_px,
                       const sd_subswath *sw, const int64_t *azimuth_start_time_us,
                       float *out_data, float *out_nesz, sd_merged_info *info);

/* ── Fused calibrate + deburst + merge ────────────────────────────────────
 * The per-IW chain of prepare_merged_scene (scene_prep.rs:598-699): deburst,
 * apply_calibration with tiff_line_origin = bursts[0].first_line, then
 * merge_subswaths, in one gather kernel per swath writing straight into the
 * merged rasters.  Call with out_data == NULL to only fill *info. */
int sd_calibrate_deburst_merge(sd_ctx *ctx, int32_t n_swaths,
                               const sd_swath_input *swaths, float *out_data,
                               float *out_nesz, sd_merged_info *info);

/* ── Terrain correction ───────────────────────────────────────────────────
 * Output grid of terrain_correction (terrain_correction.rs:1174-1216,
 * 1297-1320) without running it: fills rows, cols, origin, geotransform. */
int sd_tc_output_grid(sd_ctx *ctx, const sd_scene *scene, const sd_tc_config *cfg,
                      sd_geocoded_info *info);
/* terrain_correction (terrain_correction.rs:1245-1836).  out_data is
 * rows x cols f32; out_cos_lia / out_mask are filled when cfg->compute_lia
 * (otherwise they may be NULL).  cfg->precision selects the FP64 path
 * (reference arithmetic) or the split-precision path (SD_PRECISION_SPLIT:
 * same converged azimuth times, mask and counters; FP32 resampling,
 * facet, LIA and flattening). */
int sd_terrain_correction(sd_ctx *ctx, const sd_radar_image *image,
                          const sd_scene *scene, const sd_dem *dem,
                          const sd_geoid *geoid, const sd_geo_grid_point *grid,
                          uint64_t n_grid, const sd_tc_config *cfg,
                          float *out_data, float *out_cos_lia, uint8_t *out_mask,
                          sd_geocoded_info *info);
/* Rows [row_begin, row_end) of sd_terrain_correction's output grid
 * (row_end 0 = to the last row): the outputs hold (row_end - row_begin) x
 * cols pixels, the counters cover the band, and the band's values equal
 * those rows of the whole-grid call (each output row's solve chain starts
 * from its own LUT seed, terrain_correction.rs:1443).  This is how one
 * scene shards over GPUs by output rows without any exchange.
 * out_azimuth_time_us (may be NULL) receives the per-pixel converged times
 * as in sd_terrain_correction_with_times. */
int sd_terrain_correction_rows(sd_ctx *ctx, const sd_radar_image *image,
                               const sd_scene *scene, const sd_dem *dem,
                               const sd_geoid *geoid, const sd_geo_grid_point *grid,
                               uint64_t n_grid, const sd_tc_config *cfg,
                               uint64_t row_begin, uint64_t row_end,
                               float *out_data, float *out_cos_lia, uint8_t *out_mask,
                               int64_t *out_azimuth_time_us, sd_geocoded_info *info);
/* sd_terrain_correction plus the converged zero-Doppler azimuth time of
 * every output pixel in integer microseconds (INT64_MIN where the solve did
 * not converge, the DEM has no height or the orbit refused the time), for
 * measuring geolocation against another implementation.  No counterpart in
 * the reference (its per-pixel time is internal to the loop at
 * terrain_correction.rs:1513-1740). */
int sd_terrain_correction_with_times(sd_ctx *ctx, const sd_radar_image *image,
                                     const sd_scene *scene, const sd_dem *dem,
                                     const sd_geoid *geoid, const sd_geo_grid_point *grid,
                                     uint64_t n_grid, const sd_tc_config *cfg,
                                     float *out_data, float *out_cos_lia, uint8_t *out_mask,
                                     int64_t *out_azimuth_time_us, sd_geocoded_info *info);

/* ── Device-resident scenes and batched tiles ──────────────────────────────
 * No single counterpart in the reference: its terrain_correction
 * (terrain_correction.rs:1245-1836) geocodes one scene onto one grid per call.
 * Here a scene is uploaded once and any number of output tiles (windows of
 * any size, over any resident scene) are geocoded per batch, each tile
 * exactly as terrain_correction would geocode that tile's own grid (its rows
 * seeded from the LUT, its own per-row flat area and UTM anchors). */
typedef struct sd_scene_dev sd_scene_dev;

/* Keeps the radar image (and NESZ), DEM, geoid, state vectors, the
 * azimuth-time LUT of `grid` and an FP64 orbit table over the image's azimuth
 * span in device memory.  Host buffers are copied; device buffers are
 * borrowed (keep them alive until sd_scene_destroy).  Errors as
 * sd_terrain_correction's argument checks. */
int sd_scene_create(sd_ctx *ctx, const sd_radar_image *image, const sd_scene *scene,
                    const sd_dem *dem, const sd_geoid *geoid, const sd_geo_grid_point *grid,
                    uint64_t n_grid, sd_scene_dev **out);
/* Device bytes the scene owns (copies and orbit table). */
uint64_t sd_scene_device_bytes(const sd_scene_dev *scene);
/* Frees the scene; no batch that reads it may be in flight. */
void sd_scene_destroy(sd_scene_dev *scene);

typedef struct {
    sd_scene_dev *scene;
    sd_tc_config cfg;           /* pixel_spacing, crs and utm_zone give the tile's CRS */
    double origin_x;            /* west edge: longitude (deg) or UTM easting (m) */
    double origin_y;            /* north edge: latitude (deg) or UTM northing (m) */
    uint64_t rows, cols;
    int32_t speckle;            /* -1: none, else SD_SPECKLE_* applied after geocoding */
    int32_t speckle_window;     /* odd, 3..15 (Refined Lee: 7) */
    float enl, damping;
    /* rows x cols outputs, device or host memory (host: pinned for overlap).
     * With a speckle filter the tile is geocoded with a halo of half a
     * window on every side and filtered before cropping, so the result
     * equals the filter applied to the larger raster, then cropped. */
    float *out_data;
    float *out_cos_lia;         /* required when cfg.compute_lia */
    uint8_t *out_mask;          /* required when cfg.compute_lia */
} sd_tile;

/* Enqueues the batch on the context's stream and returns; tiles may mix
 * scenes, sizes, resampling kernels, precisions and filters.  One batch per
 * context is in flight at a time (SD_ERR_BUSY otherwise). */
int sd_tc_tiles_launch(sd_ctx *ctx, const sd_tile *tiles, uint64_t n);
/* Host delivery of a batch in flight: one copy of `bytes` from device
 * memory dev_src (normally the results' arena) to host memory host_dst
 * (pinned for an asynchronous copy), enqueued on the context's stream
 * behind the batch's kernels; the batch completes (sd_tc_tiles_poll /
 * _finish) once the copy has landed.  No reference counterpart (serving). */
int sd_tc_tiles_copy_out(sd_ctx *ctx, void *host_dst, const void *dev_src, uint64_t bytes);
/* SD_OK when the batch in flight has finished (or none is), SD_ERR_BUSY if not. */
int sd_tc_tiles_poll(sd_ctx *ctx);
/* Waits for the batch and fills infos[0..n) (counters, histogram, grid). */
int sd_tc_tiles_finish(sd_ctx *ctx, sd_geocoded_info *infos, uint64_t n);
/* sd_tc_tiles_launch + sd_tc_tiles_finish. */
int sd_tc_tiles(sd_ctx *ctx, const sd_tile *tiles, uint64_t n, sd_geocoded_info *infos);
/* Replay the tile stages as CUDA graphs of persistent kernels (captured on
 * first use per variant; work tables keep fixed addresses up to 1024 tiles). */
int sd_ctx_set_graphs(sd_ctx *ctx, int enable);
/* Allocates the context's tile scratch up front: an arena of
 * `tile_arena_bytes` plus the work tables of a 1024-tile batch, so batches
 * that fit it run without device allocations. */
int sd_ctx_reserve(sd_ctx *ctx, uint64_t tile_arena_bytes);
/* Launch shapes of the tile stages: the speckle/crop block (tx x ty
 * threads, tx >= 8, tx*ty <= 512 and a multiple of 32; default 32 x 8) and
 * the geocoding kernel: CTAs per SM of its persistent form (0 = as many as
 * fit), or -1 for one launch per tile with the job in parameter space over
 * four forked streams.  Results do not depend on them;
 * sardine_b200.autotune picks them. */
int sd_ctx_set_tile_shape(sd_ctx *ctx, int32_t speckle_tx, int32_t speckle_ty,
                          int32_t main_ctas_per_sm);

/* interpolate_orbit_and_accel (orbit.rs:498-596) at m integer-microsecond
 * times, as the terrain correction evaluates it on the GPU: out holds
 * m x {pos xyz, vel xyz, acc xyz}.  SD_ERR_TC_ORBIT when a time is outside
 * the state vectors' span or fewer than 8 vectors are given. */
int sd_orbit_states(sd_ctx *ctx, const sd_state_vector *svs, uint64_t n, const int64_t *t_us,
                    uint64_t m, double *out);

/* ── SLC ingest ───────────────────────────────────────────────────────────
 * SlcReader (slc_reader.rs:485-598) over a Sentinel-1 measurement TIFF:
 * classic TIFF, CInt16 (SampleFormat 5, 32 bits), uncompressed, one row per
 * strip, contiguous strips (the checks of parse_ifd, 268-465, in its
 * order and with its errors, SD_ERR_SLC_*).  sd_slc_open keeps the file
 * open until sd_slc_close; sd_slc_dims gives width, height and byte order. */
typedef struct sd_slc_reader sd_slc_reader;
int sd_slc_open(sd_ctx *ctx, const char *path, sd_slc_reader **out);
int sd_slc_dims(const sd_slc_reader *reader, uint32_t *width, uint32_t *height, int32_t *little_endian);
void sd_slc_close(sd_slc_reader *reader);
/* read_burst_raw (532-583): line_count rows from first_line as [I, Q]
 * int16 pairs (line_count x width x 2), in host byte order.  out may be
 * host or device memory.  Into device memory, four threads read 32 MB
 * chunks in parallel into pinned buffers the reader keeps (256 MB, freed
 * by sd_slc_close) while earlier chunks are copied on the context's
 * stream.  One read at a time per reader (it is `&mut self` in the
 * reference).  Rows past the image give SD_ERR_SLC_LINE_OUT_OF_BOUNDS,
 * failed reads SD_ERR_SLC_IO. */
int sd_slc_read_burst_raw(sd_ctx *ctx, sd_slc_reader *reader, uint64_t first_line, uint64_t line_count,
                          int16_t *out);

/* ── Pre-TC multilook ─────────────────────────────────────────────────────
 * The boxcar of apply_multilook (scene_prep.rs:1060-1160) over a merged
 * image (lines x samples, host or device): out_data/out_nesz
 * ((lines / azimuth_looks) x (samples / range_looks)) hold the f64 mean of
 * the non-NaN sigma0 of each azimuth_looks x range_looks block and of the
 * NESZ at those same pixels, NaN when all are NaN.  nesz may be NULL (then
 * out_nesz is ignored).  The geometry update (spacing x range_looks, near
 * range + (R-1)/2 spacings, azimuth start + (A-1)/2 ATI) is the caller's;
 * sardine_b200.apply_multilook does both.  Factors of 0, or larger than
 * the image, give SD_ERR_INVALID_ARGUMENT with the reference's message. */
int sd_multilook(sd_ctx *ctx, const float *data, const float *nesz, uint64_t lines, uint64_t samples,
                 uint32_t range_looks, uint32_t azimuth_looks, float *out_data, float *out_nesz);

/* ── Ground range (GRD) ───────────────────────────────────────────────────
 * to_ground_range (ground_range.rs:303-427) of a merged slant-range image
 * (lines x samples, host or device): the incidence-angle profile from each
 * sub-swath's mid-azimuth geolocation row, ground spacing = slant spacing /
 * sin(incidence), output columns every target_spacing_m of cumulative
 * ground range (linear f32 interpolation between slant columns), then the
 * f64 mean of round(target / azimuth_pixel_spacing_m) lines (NaN skipped).
 * Call with out == NULL to only fill *info (the output dimensions). */
typedef struct sd_grd_grid_point {   /* GeolocationGridPoint fields read here (types.rs:171) */
    uint32_t line;
    uint32_t pad;
    double slant_range_time_s;
    double incidence_angle_deg;
} sd_grd_grid_point;
typedef struct sd_grd_swath_grid {   /* one (SubSwathId, Vec<GeolocationGridPoint>) */
    int32_t swath_id;                 /* 1..3 for IW1..IW3 (messages only) */
    int32_t pad;
    const sd_grd_grid_point *points;
    uint64_t n_points;
} sd_grd_swath_grid;
typedef struct sd_grd_info {         /* GroundRangeImage (ground_range.rs:60-85) minus data */
    uint64_t lines, samples;
    double range_pixel_spacing_m, azimuth_pixel_spacing_m;
    uint64_t range_looks, azimuth_looks;
} sd_grd_info;
int sd_to_ground_range(sd_ctx *ctx, const float *data, uint64_t lines, uint64_t samples,
                       double near_slant_range_time_s, double range_pixel_spacing_s,
                       double range_pixel_spacing_m, const sd_grd_swath_grid *grids, int32_t n_grids,
                       double target_spacing_m, double azimuth_pixel_spacing_m, float *out,
                       sd_grd_info *info);

/* ── TOPS deramping (InSAR) ───────────────────────────────────────────────
 * deramp_subswath (insar/deramp.rs:114-210) of a debursted sub-swath iq
 * (lines x samples CInt16 pairs, host or device): out (lines x samples
 * complex f32 pairs, same kind of memory) = iq * exp(-j phi), phi =
 * 2 pi f_DC(tau) t_az, tau = slant_range_time_s + (c + valid_sample_offset)
 * * 2 range_pixel_spacing_m / c, t_az = l * azimuth_time_interval_s and
 * f_DC = a0 + a1 (tau - t0) + a2 (tau - t0)^2 with (a0, a1, a2, t0)
 * interpolated linearly in azimuth time between the two estimates around
 * the line (interp_dc_poly, deramp.rs:227-276; first/last estimate outside
 * them).  burst_start_us is the azimuth time of line 0; swath_id (1..3 for
 * IW1..IW3) only names the swath in messages.
 * Errors: SD_ERR_INSAR_NO_DC_ESTIMATES, SD_ERR_INSAR_AZIMUTH_TIME_BEFORE_DC
 * (a line more than 2 s before the first estimate). */
typedef struct sd_dc_estimate {      /* DcEstimate (types.rs:206-213) */
    int64_t azimuth_time_us;         /* UTC, microseconds (any fixed epoch shared with burst_start_us) */
    double t0_s;
    double data_dc_poly[3];
} sd_dc_estimate;
int sd_deramp_subswath(sd_ctx *ctx, const int16_t *iq, uint64_t lines, uint64_t samples,
                       uint64_t valid_sample_offset, double slant_range_time_s, double range_pixel_spacing_m,
                       double azimuth_time_interval_s, const sd_dc_estimate *estimates, uint64_t n_estimates,
                       int64_t burst_start_us, int32_t swath_id, float *out);

/* resample_secondary (insar/coreg.rs:230-264): out (lines x samples complex
 * f32) at reference pixel (l, c) is the bilinear sample (coreg.rs:428-456;
 * f32 weights, zero outside) of sec (sec_lines x sec_samples complex f32) at
 * (l + P_az(l, c), c + P_rg(l, c)), P(l, c) = p0 + p1 l + p2 c + p3 l^2 +
 * p4 l c + p5 c^2 (CoregPoly, coreg.rs:73-90).  Host or device memory. */
int sd_resample_secondary(sd_ctx *ctx, const float *sec, uint64_t sec_lines, uint64_t sec_samples,
                          uint64_t lines, uint64_t samples, const double *az_poly, const double *rg_poly,
                          float *out);

/* compute_coreg_offsets (insar/coreg.rs:128-223): a 20 x 50 grid of reference
 * pixels ((i+1) lines / 21, (j+1) samples / 51), each forward-geocoded to the
 * WGS84 ellipsoid (ecef_from_slant_range_doppler, 20 iterations, 1 mm),
 * then solve_zero_doppler on the secondary orbit from sec_first_us (20
 * iterations, 1e-9 s) to its secondary line and column (column offset
 * sec_first_sample); failed points are skipped.  The degree-2 fits of the
 * line and column offsets (normal equations, Gaussian elimination with
 * partial pivoting) fill *out.  The grid runs on the device, the fit on
 * the host.  SD_ERR_INSAR_COREG_GRID_TOO_SMALL with fewer than 6 points or
 * a singular system. */
typedef struct sd_coreg_result {     /* CoregResult (coreg.rs:102-109) */
    double az_poly[6];
    double rg_poly[6];
    double fit_residual_rms;
    uint64_t n_valid;
} sd_coreg_result;
int sd_coreg_offsets(sd_ctx *ctx, const sd_state_vector *ref_orbit, uint64_t n_ref, int64_t ref_first_us,
                     uint64_t ref_lines, uint64_t ref_samples, uint64_t ref_valid_sample_offset,
                     double ref_azimuth_time_interval_s, double ref_slant_range_time_s,
                     double ref_range_pixel_spacing_m, const sd_state_vector *sec_orbit, uint64_t n_sec,
                     int64_t sec_first_us, double sec_azimuth_time_interval_s, double sec_slant_range_time_s,
                     double sec_range_pixel_spacing_m, uint64_t sec_first_sample, sd_coreg_result *out);

/* form_interferogram (insar/interferogram.rs:165-398) of a co-registered
 * pair ref, sec (lines x samples complex f32, host or device): per pixel the
 * flat-earth phase (4 pi / wavelength) (R_ref - R_sec) of the point on the
 * WGS84 ellipsoid at the reference range in the zero-Doppler plane of the
 * reference state at line time ref_first_us + trunc(l * ATI * 1e6) us
 * (ecef_from_slant_range_doppler, coreg.rs:280-362; 0 where it does not
 * converge), igram = ref conj(sec) exp(+j phi_flat), then over the window of
 * rows l -+ az_looks/2 and columns c -+ rg_looks/2 (clamped to the image)
 * coherence = min(|sum igram| / sqrt(sum |ref|^2 sum |sec|^2), 1) (0 when the
 * powers sum to 0) and, when phase != NULL, phase = atan2 of the summed
 * igram.  Errors: SD_ERR_INSAR_INVALID_WINDOW_SIZE (a zero window),
 * SD_ERR_INSAR_ORBIT (a line time outside either orbit). */
int sd_form_interferogram(sd_ctx *ctx, const float *ref, const float *sec, uint64_t lines, uint64_t samples,
                          uint64_t valid_sample_offset, double slant_range_time_s, double range_pixel_spacing_m,
                          double azimuth_time_interval_s, const sd_state_vector *ref_orbit, uint64_t n_ref,
                          int64_t ref_first_us, const sd_state_vector *sec_orbit, uint64_t n_sec,
                          double wavelength_m, uint32_t az_looks, uint32_t rg_looks, float *coherence,
                          float *phase);

/* ── Output: dB conversion and Cloud-Optimised GeoTIFF ───────────────────
 * to_db_inplace (export.rs:59-99) on data[0..n) in place (host or device
 * memory): NaN stays NaN; v <= noise_floor_linear (and any v <= 0) becomes
 * NaN and is counted as noise-masked; every other value becomes
 * 10 log10(v) (f32).  counts (may be NULL) receives {converted,
 * noise_masked}.  stats (may be NULL) receives compute_db_stats
 * (run.rs:63-97) of the converted raster: {min, max, mean, median} of the
 * finite values, the mean from an f64 sum, the median of every
 * max(n_finite / 100000, 1)-th finite value; NaN when none is finite.
 * SD_ERR_EXPORT_INVALID_NOISE_FLOOR when noise_floor_linear < 0. */
int sd_to_db(sd_ctx *ctx, float *data, uint64_t n, float noise_floor_linear, uint64_t *counts,
             float *stats);

/* dB output fused into the producing kernel: after
 * sd_ctx_set_db_output(ctx, 1, noise_floor_linear), sd_terrain_correction
 * (and its _rows/_with_times forms) and sd_speckle on this context write
 * their sigma0/gamma0 (resp. filtered) raster in dB exactly as sd_to_db
 * would convert it afterwards (to_db_inplace, export.rs:59-99, as run.rs:
 * 395-403 applies it to the last stage's output), so the separate
 * read-modify-write pass over the raster disappears.  sd_ctx_db_result then
 * returns that call's {converted, noise_masked} counts and the
 * compute_db_stats (run.rs:63-97) {min, max, mean, median} of the raster it
 * wrote (of the band, for sd_terrain_correction_rows).  enable = 0 restores
 * linear output.  SD_ERR_EXPORT_INVALID_NOISE_FLOOR when noise_floor_linear
 * < 0.  No reference counterpart: the reference converts in a separate
 * pass. */
int sd_ctx_set_db_output(sd_ctx *ctx, int32_t enable, float noise_floor_linear);
/* counts: {converted, noise_masked}; stats: {min, max, mean, median}.
 * SD_ERR_INVALID_ARGUMENT if no call with dB output has completed. */
int sd_ctx_db_result(sd_ctx *ctx, uint64_t *counts, float *stats);

/* Debug builds (compiled with -DSD_BOUNDS_CHECK=1) test every radar-image
 * and DEM gather of the terrain-correction kernels against the buffer's
 * extent, skip an access outside it and record the first one.  word[0..4):
 * {site (1 radar image, 2 DEM; 0 = none since the last call), index,
 * extent, 1 if this build has the checks else 0}; reading clears the
 * record.  No reference counterpart (the reference relies on Rust's bounds
 * checks). */
int sd_debug_bounds(sd_ctx *ctx, uint64_t *word);

/* downsample_2x (export.rs:362-392): dst ((cols+1)/2 x (rows+1)/2) holds the
 * f64 mean of the non-NaN pixels of each 2x2 patch of src, NaN when all
 * are NaN.  The overview step of sd_write_cog. */
int sd_downsample_2x(sd_ctx *ctx, const float *src, uint64_t cols, uint64_t rows, float *dst);

/* write_cog_with_crs (export.rs:329-355, writer 417-760): a single-band
 * Float32 COG of data (rows x cols, host or device) at `path`: overview
 * levels by downsample_2x down to one tile, IFDs coarsest first, 17 tags
 * each, GeoKeys of crs (SD_CRS_*, utm_zone 1..60 for UTM), tiles of
 * tile_size^2 padded with NaN, BigTIFF when rows*cols*4 exceeds 4 GiB.
 * Overviews and tiles are built on the device; the host writes the file.
 * Errors: SD_ERR_EXPORT_INVALID_GEOTRANSFORM, SD_ERR_EXPORT_INVALID_TILE_SIZE
 * (a power of two in [64, 4096]), SD_ERR_EXPORT_IO. */
int sd_write_cog(sd_ctx *ctx, const char *path, const float *data, uint64_t cols, uint64_t rows,
                 const double *geotransform, int32_t crs, int32_t utm_zone, uint32_t tile_size);

/* ── Diagnostics ──────────────────────────────────────────────────────────
 * Runs an FP64 FMA-chain kernel for about `iters` dependent FMAs per thread
 * over the whole device and returns the achieved FP64 TFLOP/s. */
int sd_measure_fp64_peak(sd_ctx *ctx, int32_t iters, double *tflops);
int sd_measure_fp32_peak(sd_ctx *ctx, int32_t iters, double *tflops);

/* Correctly rounded sin and cos (the device's copy of the function the
 * terrain correction takes its target ECEF sines and cosines from) of n
 * doubles in device memory; no counterpart in the reference, which calls the
 * platform libm (geodesy.rs:42-45). */
int sd_cr_sincos(sd_ctx *ctx, const double *x, uint64_t n, double *s, double *c);

#ifdef __cplusplus
}
#endif
#endif /* SARDINE_B200_H */
