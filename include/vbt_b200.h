/*
 * vbt_b200.h -- C-ABI of the B200 (sm_100a) decode path for VBTPACK4 assets.
 *
 * Plain C types only: pointers, sizes, and an opaque asset handle.  Device pointers are CUDA
 * device addresses on the asset's device; `stream` is a cudaStream_t (NULL = legacy default).
 * Every call returns a status (VBT_STATUS_*); a message for the last failure on the calling
 * thread is available from vbt_last_error().  There is no CPU execution path: a process without
 * a usable CUDA device gets VBT_STATUS_CUDA from every decode call.
 *
 * The reference interfaces each call replaces are cited as file:line inside the VBT project.
 */
#ifndef VBT_B200_H
#define VBT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (1..13 mirror the reference's std::runtime_error messages) ---- */
#define VBT_STATUS_OK 0
#define VBT_STATUS_LEAF_TOO_SMALL 1       /* "render temporal leaf bytes too small" */
#define VBT_STATUS_PREFIX_MISSING 2       /* "render temporal leaf prefix missing" */
#define VBT_STATUS_LEAF_SHORT 3           /* "render temporal leaf shorter than computed layout" */
#define VBT_STATUS_SHELL_OCC_OOB 4        /* "render temporal shell occupancy is out of bounds" */
#define VBT_STATUS_SHELL_GROUP_PREFIX 5   /* "render temporal shell group prefix is inconsistent" */
#define VBT_STATUS_SHELL_NO_ACTIVE 6      /* "render temporal shell mode contains no active voxels" */
#define VBT_STATUS_SHELL_RESIDUAL_OOB 7   /* "render temporal shell residual stream is out of bounds" */
#define VBT_STATUS_SHELL_TRAILING 8       /* "render temporal shell leaf contains trailing bytes" */
#define VBT_STATUS_CONTROL_INDEX 9        /* "render temporal control index out of range" */
#define VBT_STATUS_STREAM_OOB 10          /* "render temporal stream decode out of bounds" */
#define VBT_STATUS_DECODE_OOB 11          /* "render temporal decode out of bounds" / std::out_of_range */
#define VBT_STATUS_KEY_RANGE_OOB 12       /* "render temporal keyframe range out of bounds" */
#define VBT_STATUS_KEY_INDEX 13           /* "render temporal keyframe index out of range" */
#define VBT_STATUS_WAIT_TIMEOUT 30        /* a bounded device-side wait gave up (no hang) */
#define VBT_STATUS_INVALID_ARGUMENT 40
#define VBT_STATUS_FILE 41                /* the VBTPACK4 reader rejected the file (message set) */
#define VBT_STATUS_CUDA 42                /* CUDA runtime error or no usable device (message set) */
#define VBT_STATUS_LIMIT 43               /* request exceeds a fixed capacity of the call */
#define VBT_STATUS_UNSUPPORTED 44         /* a leaf mode the call does not cover (recorded per leaf) */

typedef struct vbt_asset vbt_asset;

/* VBTPACK4 header fields; replaces vbt::render::VbtFileHeader (render/src/vbt_file.h:10-23). */
typedef struct {
    uint32_t version, width, height, depth, frames, leaf_size, coarse_resolution, max_coarse_keep,
        leaf_count, profile_type, coarse_ac_scale_count;
} vbt_header;

typedef struct {
    vbt_header header;
    uint32_t leaf_count_x, leaf_count_y, leaf_count_z;
    uint32_t active_leaf_count;  /* from the last page-table build (synchronised read) */
    uint64_t payload_words;
    uint64_t device_bytes;       /* device memory held by the asset */
    int device;
} vbt_asset_info;

const char* vbt_status_string(int status);
const char* vbt_last_error(void);
int vbt_device_count(void);

/* Validate a whole VBTPACK4 file image with the reader's rules and messages
 * (replaces vbt::render::loadVbtFile's checks, render/src/vbt_file.cpp:39-206). */
int vbt_validate_file_image(const void* bytes, uint64_t len, vbt_header* out_header);

/* Load an asset and keep it resident on `device`: offsets, payload, scales, leaf table, page
 * table.  The page table is built once during the call.  Replaces loadVbtFile
 * (render/src/vbt_file.cpp:109-210) + the Studio's upload (VBTStudio/frontend/src/
 * volume_renderer.cpp:1593-1608). */
int vbt_asset_open(const char* path, int device, vbt_asset** out_asset);
int vbt_asset_create(const void* file_bytes, uint64_t len, int device, vbt_asset** out_asset);
int vbt_asset_destroy(vbt_asset* asset);
/* Re-upload a file image with the same header and sizes into the asset's resident buffers,
 * asynchronously on `stream` (host memory should be pinned), then re-walk the leaves and redo the
 * per-asset key-order analysis on the same stream.  Leaf offsets are checked on the device by the
 * walker (a leaf whose offsets leave the payload gets VBT_STATUS_DECODE_OOB). */
int vbt_asset_upload(vbt_asset* asset, const void* file_bytes, uint64_t len, void* stream);
int vbt_asset_get_info(vbt_asset* asset, vbt_asset_info* out_info);

/* Kernel (a): active-leaf page table (compact[leaf] = ascending rank among non-EMPTY leaves,
 * 0xFFFFFFFF for EMPTY), the Studio's page-table shader
 * (VBTStudio/frontend/shaders/vbt_active_index.comp:28-57).  The payload walker, which replaces
 * parseRenderTemporalPackedLeaf (src/render_temporal_payload.cpp:234-311) per leaf, runs when the
 * payload is uploaded (vbt_asset_create / vbt_asset_upload) and leaves a per-leaf table; this
 * call compacts that table's active flags.  Asynchronous on `stream`. */
int vbt_build_page_table(vbt_asset* asset, void* stream);
/* Device views of the page table: compact[leaf_count], active_list[rank] = leaf, and the
 * device-resident active count (one uint32). */
int vbt_page_table_device(vbt_asset* asset, const uint32_t** d_compact, const uint32_t** d_active_list,
                          const uint32_t** d_active_count);
/* Synchronous host copy of the page table (compact must hold leaf_count entries). */
int vbt_get_page_table(vbt_asset* asset, uint32_t* compact, uint32_t* active_count);
/* Synchronous host copy of the 32-byte leaf-table rows (8 uint32 per leaf). */
int vbt_get_leaf_table(vbt_asset* asset, uint32_t* rows);

/* Kernel (b): current-frame voxel cache for `nframes` (<= 128) frames in one launch:
 * d_out[f * frame_stride + rank * 512 + (lz*8 + ly)*8 + lx].  Voxels outside a boundary leaf's
 * extent are 0.  Values equal decodeFrameToDense (render/src/render_smoke_vbt_bench_main.cpp:
 * 389-452) voxel for voxel; the Studio cache it replaces is vbt_cache.comp:176-294.
 * `grid` = CTAs of the persistent launch (0 = one wave of the device). */
int vbt_decode_cache(vbt_asset* asset, const int* frames, int nframes, float* d_out, uint64_t frame_stride,
                     int grid, void* stream);
/* The reference Studio's control cache (VBTStudio/frontend/shaders/vbt_cache.comp:168-236), for
 * consumers written against it: d_out[f * frame_stride + rank * 576 + slot] over the active leaves
 * of the current page table (vbt_build_page_table first) and frames[0..nframes) (clamped as the
 * reference clamps, 1..128 frames).  Slot s < 64 holds coarse control s; from slot 64 on, the fine
 * grid's controls (FINE6) or the Mode2 shell residual controls; other slots hold 0.  Values are
 * the reference CPU decoder's (decodeRenderTemporalControlValue, src/render_temporal_decode.cpp:
 * 304-356); render-temporal assets only. */
int vbt_decode_control_cache(vbt_asset* asset, const int* frames, int nframes, float* d_out, uint64_t frame_stride,
                             void* stream);
/* ---- Ray sampling from the control cache ------------------------------------------------------
 * The Studio's sampler (VBTStudio/frontend/shaders/vbt_sample.comp:322-622) as plain CUDA, one
 * thread per ray, results in a device buffer.  Rays and results are the shader's SmokeRayPacked
 * and VbtSampleResult.  d_controls is the control cache of frame params->frame_index
 * (vbt_decode_control_cache) over the current page table.  render_mode 0 accumulates the field
 * along each ray over step_count steps (surface_model != 0: into 8 depth bins, primary then
 * auxiliary); render_mode 1 traces the surface phi = surface_iso (primary = normal, hit t or -1;
 * auxiliary = thickness, floor flag, floor shadow, |n . -dir|).  Single precision, each operation
 * rounded, GLSL mix / min / max / clamp; round() rounds halves away from zero; a coarse grid over
 * 64 controls is decoded from the payload.  Render-temporal assets; both buffers 16-byte aligned. */
typedef struct {
    float origin_tmin[4]; /* origin x, y, z and t_min */
    float dir_tmax[4];    /* direction x, y, z and t_max */
} vbt_ray;
typedef struct {
    float primary[4];
    float auxiliary[4];
} vbt_sample_result;
typedef struct {
    uint32_t step_count;
    int32_t frame_index;
    float bbox_min[3];         /* world position of voxel (0, 0, 0) */
    uint32_t render_mode;      /* 0 density accumulation, 1 level-set surface */
    float voxel_size, background_value, surface_iso, surface_epsilon_voxels, surface_normal_step, max_step_voxels;
    uint32_t surface_model;
    float floor_height;
    uint32_t shadow_steps;
    uint32_t up_axis;          /* the shader's `padding`: 2 = z up for the floor plane and key light */
} vbt_sample_params;
int vbt_sample_rays(vbt_asset* asset, const float* d_controls, const vbt_sample_params* params, const vbt_ray* d_rays,
                    uint32_t n, vbt_sample_result* d_out, void* stream);
/* The render tree's smoke sampler (render/shaders/vbt_smoke_sample.comp:124-336) as plain CUDA, one
 * thread per ray: d_out[i] = the sum of params->step_count density samples along ray i at
 * params->frame_index, each decoded straight from the payload (coarse stream, plus the FINE6 stream;
 * Mode2 leaves contribute their coarse stream, as in the shader) with the shader's own control
 * decode, whose lerp is mix(previous, next, w).  Uses step_count, frame_index and bbox_min only;
 * no control cache.  Render-temporal assets; rays 16-byte aligned. */
int vbt_smoke_sample_rays(vbt_asset* asset, const vbt_sample_params* params, const vbt_ray* d_rays, uint32_t n,
                          float* d_out, void* stream);

/* ---- VBTPACK4 writer, payload half ------------------------------------------------------------
 * What writeRenderTemporalProbeFile (src/render_temporal_kf_probe_main.cpp:2561-2585) builds on
 * the host, on the GPU: leaf_count packed leaf blocks (any byte lengths, 0 included) concatenated
 * in d_blocks, block i at bytes [d_block_offsets[i], d_block_offsets[i + 1]) -> d_offsets
 * (leaf_count + 1 word offsets) and d_payload (each block padded with zero bytes to whole words, in
 * leaf order).  *total_words = d_offsets[leaf_count]; VBT_STATUS_LIMIT when it exceeds
 * payload_capacity_words or 2^32 words (d_payload is then not written).  The file is the 52-byte
 * header, d_offsets and d_payload.  Synchronises `stream` once (to read the payload size). */
int vbt_pack_payload(const uint8_t* d_blocks, const uint64_t* d_block_offsets, uint32_t leaf_count, uint32_t* d_offsets,
                     uint32_t* d_payload, uint64_t payload_capacity_words, uint64_t* total_words, void* stream);

/* ---- VBTPACK4 writer, leaves from control streams -----------------------------------------------
 * packRenderTemporalControlStream (src/render_temporal_decode.cpp:201-264) for every stream and
 * buildRenderTemporalPackedLeafBytes (src/render_temporal_payload.cpp:199-232; the Mode2 shell
 * overload :348-386), 4-byte aligned as the encoder writes them, for leaf_count leaves at once,
 * straight into the payload: d_offsets (leaf_count + 1 word offsets) and d_payload, as
 * vbt_pack_payload lays them out.  Per leaf, a vbt_leaf_streams names its packed header word
 * (packRenderTemporalHeader: mode, codecs, resolutions), its prefix, and where its streams' rows
 * start in the shared arrays:
 *   d_descriptors  one RenderTemporalControlDescriptor per control row (keyStart | keyCount << 16 |
 *                  reserved << 24), control_rows rows
 *   d_bins         8 bytes per control row, the stream's time-bin index (4-bin Mode2 residual
 *                  streams use the first 4)
 *   d_key_frames / d_key_values  key_rows keyframes (frame, value); FP16 streams store the value
 *                  as renderTemporalFloatToHalfBits(value)
 *   d_occupancy    occupancy_rows 80-byte Mode2 shell occupancy sections (4-byte aligned)
 * A stream has resolution^3 controls (the Mode2 residual stream: the occupancy's active voxels),
 * 8 time bins (Mode2 residual: 4) and the prefix's keyframe count.  Invalid streams
 * (validateRenderTemporalControlStreamData, with the leaf's max_local as maxBinLocalKeys), FP16
 * frames above 255 and rows outside the arrays give VBT_STATUS_INVALID_ARGUMENT with the
 * reference's message and the lowest failing leaf; nothing is written then.  Synchronises
 * `stream` once (to read the payload size). */
typedef struct {
    uint32_t header;                               /* packRenderTemporalHeader word */
    uint16_t coarse_keyframes, fine_keyframes;     /* RenderTemporalPackedLeafPrefix */
    uint32_t coarse_control, coarse_key;           /* first control row / keyframe of the coarse stream */
    uint32_t fine_control, fine_key;               /* FINE6 stream, or the Mode2 shell residual stream */
    uint32_t occupancy;                            /* Mode2: row of the leaf's occupancy section */
    uint8_t coarse_max_local, fine_max_local;      /* the streams' maxBinLocalKeys */
    uint8_t pad[2];
} vbt_leaf_streams;
int vbt_pack_leaves(const vbt_leaf_streams* d_leaves, uint32_t leaf_count, const uint32_t* d_descriptors,
                    const uint8_t* d_bins, uint64_t control_rows, const uint16_t* d_key_frames,
                    const float* d_key_values, uint64_t key_rows, const uint8_t* d_occupancy, uint64_t occupancy_rows,
                    uint32_t* d_offsets, uint32_t* d_payload, uint64_t payload_capacity_words, uint64_t* total_words,
                    void* stream);

/* ---- Encoder keyframe pass ---------------------------------------------------------------------
 * The per-voxel body of the reference encoder's leaf loop (src/render_temporal_kf_probe_main.cpp:
 * 619-659) over `series` independent series of `frames` finite values, value t of series s at
 * d_values[t * frame_stride + s * series_stride] in either of RawVolume4D's orders
 * (src/raw_volume.cpp:58-75): frame-major, series_stride = 1 and frame_stride >= series (s =
 * (z*Y + y)*X + x, frame_stride = X*Y*Z), or time-fastest, frame_stride = 1 and series_stride >=
 * frames; other layouts are VBT_STATUS_INVALID_ARGUMENT.  The background test (max(0, values) <
 * bg_threshold, when bg_threshold >= 0),
 * detectDensityKeyFrames (:2080-2167) and reconstructFromKeys (:2169-2201).
 *   d_key_mask   word-major key sets: bit t % 32 of d_key_mask[(t / 32) * series + s]
 *   d_key_count  the count the encoder adds up: the keys, or 1 for a background-zeroed series
 *   d_flags      bit 0 background-zeroed (no keys, reconstruction 0); bit 1 usedCutoffProtect
 *   d_recon      optional, the reconstruction in the input's layout
 *   d_err2       optional, the series' squared error summed over frames in frame order
 *   d_totals     optional, overwritten: the leaf loop's totals (totalKeyframes, maxKeyframes,
 *                temporalProtectedSeries, backgroundZeroedVoxels, and the squared error, whose
 *                summation order differs from the reference's running sum)
 * Everything but d_totals->err2 equals the reference bit for bit.  frames <= 1024 and series < 2^36
 * (VBT_STATUS_LIMIT beyond). */
typedef struct {
    float eps_abs, eps_rel, gamma_delta, render_cutoff, cutoff_band;   /* DensityTemporalProfile, :81-95 */
    uint32_t cutoff_temporal_protect, iso_surface_protect;
    float iso_value, iso_band;
    double bg_threshold;   /* :477, bgZeroRatio * cutoff (formed in float); < 0 disables the test */
} vbt_keyframe_profile;
typedef struct {
    uint64_t total_keys, protected_series, background_series;
    uint32_t max_keys, pad;
    double err2;
} vbt_keyframe_totals;
int vbt_detect_keyframes(const float* d_values, uint64_t series, uint32_t frames, uint64_t frame_stride,
                         uint64_t series_stride, const vbt_keyframe_profile* profile, uint32_t* d_key_mask, uint32_t* d_key_count,
                         uint8_t* d_flags, float* d_recon, double* d_err2, vbt_keyframe_totals* d_totals,
                         void* stream);
/* The encoder's coarse control fitting (src/render_temporal_kf_probe_main.cpp:705-729) for
 * leaf_count leaves of a frame-major reconstruction d_recon (the keyframe pass's, value t of voxel
 * (z*height + y)*width + x at d_recon[t * frame_stride + voxel]): per listed leaf (index
 * (bz*lcy + by)*lcx + bx of the 8^3 leaf grid), its 4^3 controls sampled at controlCoords(4)
 * (sampleLeafBufferAtFractional, :2203-2237), keyed with detectDensityKeyFrames under
 * control_profile (no background test) and appended as appendControlSequenceToStream
 * (:2361-2399) appends them with 8 time bins.  Outputs per listed leaf i: d_desc[i*64 + c]
 * (keyStart | keyCount << 16 | reserved << 24), d_bins[(i*64 + c)*8 + b], keyframes from
 * d_key_frames / d_key_values[i * 64 * frames] on, d_key_count[i] (0xFFFFFFFF for a leaf index
 * outside the grid), d_required_max_local[i], and optionally the fitted grid
 * d_grid[(i*64 + c) * frames + t] (reconstructFromKeys).  These are the stream arrays
 * vbt_pack_leaves reads (bin rows 8 bytes apart).  No reference counterpart as a function: the
 * reference fits inside its leaf loop. */
int vbt_coarse_fit(const float* d_recon, uint32_t width, uint32_t height, uint32_t depth, uint32_t frames,
                   uint64_t frame_stride, const uint32_t* d_leaves, uint32_t leaf_count,
                   const vbt_keyframe_profile* control_profile, uint32_t* d_desc, uint8_t* d_bins,
                   uint16_t* d_key_frames, float* d_key_values, uint32_t* d_key_count, uint8_t* d_required_max_local,
                   float* d_grid, void* stream);
/* The encoder's FINE6 residual fitting (src/render_temporal_kf_probe_main.cpp:815-850) for the
 * listed leaves: as vbt_coarse_fit for the 6^3 controls at controlCoords(6), each series the leaf's
 * sampled reconstruction minus the fitted coarse grid (d_coarse_grid[(i*64 + c) * frames + t],
 * vbt_coarse_fit's d_grid for the same leaves) sampled at the same position
 * (sampleControlGridValue, :2240-2286).  Outputs per listed leaf i: d_desc[i*216 + c],
 * d_bins[(i*216 + c)*8 + b], keyframes from d_key_frames / d_key_values[i * 216 * frames] on,
 * d_key_count[i], d_required_max_local[i] and optionally d_grid[(i*216 + c) * frames + t]. */
int vbt_fine6_fit(const float* d_recon, uint32_t width, uint32_t height, uint32_t depth, uint32_t frames,
                  uint64_t frame_stride, const uint32_t* d_leaves, uint32_t leaf_count,
                  const vbt_keyframe_profile* control_profile, const float* d_coarse_grid, uint32_t* d_desc,
                  uint8_t* d_bins, uint16_t* d_key_frames, float* d_key_values, uint32_t* d_key_count,
                  uint8_t* d_required_max_local, float* d_grid, void* stream);
/* The encoder's Mode2 shell stage (src/render_temporal_kf_probe_main.cpp:930-1025) for the listed
 * leaves: the shell voxels (level set: |value| <= surface_band, |coarse| <= guard_band or a sign
 * change at some frame; otherwise value >= shell_cut), each one's residual over the fitted coarse
 * grid keyed under control_profile (level sets add addIsoSurfaceKeyFrames at 0 +- temporal_band,
 * :2051-2078) and appended in voxel order to a 4-bin stream with its reconstructFromKeys values.
 * Outputs per listed leaf i: the 80-byte occupancy section d_occupancy[i*80], d_desc[i*512 + a],
 * d_bins[(i*512 + a)*8 + b] (first 4 bytes), keyframes from d_key_frames / d_key_values
 * [i * 512 * frames] on, d_key_count[i], d_active[i] (shell voxels) and d_required_max_local[i]. */
int vbt_shell_fit(const float* d_recon, uint32_t width, uint32_t height, uint32_t depth, uint32_t frames,
                  uint64_t frame_stride, const uint32_t* d_leaves, uint32_t leaf_count,
                  const vbt_keyframe_profile* control_profile, const float* d_coarse_grid, int levelset,
                  float surface_band, float guard_band, float temporal_band, float shell_cut, uint8_t* d_occupancy,
                  uint32_t* d_desc, uint8_t* d_bins, uint16_t* d_key_frames, float* d_key_values,
                  uint32_t* d_key_count, uint32_t* d_active, uint8_t* d_required_max_local, void* stream);
/* The encoder's density route (src/render_temporal_kf_probe_main.cpp:1105-1245 with
 * routeRenderTemporalLeaf, src/render_temporal_route.cpp:27-66) per listed leaf: d_mode[i] = 3
 * (FINE6) or 1 (GRID4) from the raw field d_raw (frame-major) on the encoder's sampling lattice and
 * the fitted coarse and FINE6 grids (d_grid of vbt_coarse_fit / vbt_fine6_fit); peak = the field's
 * max - min (at least 1e-6), visible_lo / visible_hi = render cutoff -/+ its band. */
int vbt_route_density(const float* d_raw, uint32_t width, uint32_t height, uint32_t depth, uint32_t frames,
                      uint64_t frame_stride, const uint32_t* d_leaves, uint32_t leaf_count, const float* d_coarse_grid,
                      const float* d_fine_grid, double peak, double visible_lo, double visible_hi, uint8_t* d_mode,
                      void* stream);
/* Self-check of the division the keyframe pass uses for alpha = a / b (no reference counterpart):
 * every 1 <= b <= b_max, 0 <= a <= b against the IEEE quotient on `device`; result[0] = mismatches,
 * result[1] = (b << 16 | a) of the first, or all ones. */
int vbt_selftest_keyframe_division(uint32_t b_max, uint64_t* result, int device);

/* Plain per-leaf launch (one CTA per leaf of the grid, one frame), for comparison. */
int vbt_decode_cache_plain(vbt_asset* asset, int frame, float* d_out, void* stream);
/* Dense frames d_out[f * X*Y*Z + (z*Y + y)*X + x] (decodeFrameToDense /
 * reconstructScientificFrameCpu, render/src/scientific_decode.cpp:361-409). */
int vbt_decode_frames(vbt_asset* asset, const int* frames, int nframes, float* d_out, int grid, void* stream);

/* Kernel (c): point queries, d_xyzt = n x (x, y, z, t) uint32, 16-byte aligned.  Render family:
 * the voxel of decodeFrameToDense(t); scientific: decodeScientificValueAtCpu
 * (render/src/scientific_decode.cpp:335-359). */
int vbt_query_points(vbt_asset* asset, const uint32_t* d_xyzt, uint64_t n, float* d_out, void* stream);
/* z-slice over frames [t0, t1): d_out[(t - t0) * X*Y + y*X + x]. */
int vbt_query_slice(vbt_asset* asset, uint32_t z, int t0, int t1, float* d_out, void* stream);

/* Synchronise `stream` and return the first decode error recorded on the asset since the last
 * call (lowest failing leaf; *bad_leaf set), then clear it. */
int vbt_asset_sync_status(vbt_asset* asset, void* stream, uint32_t* bad_leaf);

/* Host-buffer calls (end-to-end: copies in, kernels, copies out, synchronised). */
int vbt_query_points_host(vbt_asset* asset, const uint32_t* xyzt, uint64_t n, float* out, void* stream);
int vbt_decode_frames_host(vbt_asset* asset, const int* frames, int nframes, float* out, void* stream);

/* Scalar decode of controls of one control stream already in device memory, one value per
 * (control index, frame) pair, with every check of decodeRenderTemporalControlValue
 * (src/render_temporal_decode.cpp:304-356); d_status[i] receives 0 or the VBT_STATUS code. */
int vbt_decode_control_values(const uint8_t* d_stream, uint32_t stream_bytes, uint32_t codec, uint32_t control_count,
                              uint32_t time_bins, uint32_t keyframe_count, int align4, int total_frames,
                              const uint32_t* d_control_index, const int32_t* d_frame, uint64_t n, float* d_out,
                              int32_t* d_status, void* stream);

/* Active-leaf page table with no allocation of any kind, for callers that must not have a library
 * allocate device memory (a renderer or plugin host that hands out all buffers from its own pool;
 * a frame loop that cannot afford cudaMalloc's device synchronisation).  No counterpart in the
 * reference.  Inputs are the asset's offsets (leaf_count + 1 words) and payload words already in
 * device memory; outputs are compact[leaf_count], active_list[leaf_count] and *active_count, with
 * the same values as vbt_build_page_table / vbt_get_page_table (0xFFFFFFFF in *active_count means a
 * bounded device-side wait gave up).  Scratch is a fixed 512 KiB array inside the library, held by
 * every GPU that loads it, so leaf_count is limited to 16,777,216 (VBT_STATUS_LIMIT beyond).  The
 * first call on a device looks up that array's device address (for the device's primary context;
 * after cudaDeviceReset the entry point must not be called again on that device) and should come
 * before any stream capture.  profile_type above 2 is VBT_STATUS_INVALID_ARGUMENT, as the reader
 * rejects it.  All calls share the array: calls whose kernels overlap on the GPU race. */
int vbt_build_page_table_noalloc(const uint32_t* d_offsets, const uint32_t* d_payload, uint64_t payload_words,
                                 uint32_t leaf_count, uint32_t profile_type, uint32_t* d_compact,
                                 uint32_t* d_active_list, uint32_t* d_active_count, void* stream);

/* ---- (d) Window decode on the tensor cores -----------------------------------------------------
 * No counterpart in the reference.  Scientific assets (profile 2): the current-frame cache of
 * frames [t0, t0 + n), n <= 64, d_out[f * frame_stride + leaf * 512 + voxel] as vbt_decode_cache,
 * computed per leaf as one contraction S(512 x 64) . C(64 x n) on tcgen05 tensor cores: S = the
 * coarse trilinear weights (343 S is an integer matrix, exact in BF16), C = the coarse controls at
 * the window's frames (the DCT-II sum of scientific_decode.cpp:82-97, in FP32) split into three
 * BF16 terms; FP32 accumulation in tensor memory; the sparse-event residual and the DenseGrid
 * residual (per-frame BFP grid or DCT temporal basis, scientific_decode.cpp:125-233) are added
 * exactly as the per-frame path does.  Values are not bit-identical to the reference;
 * vbt_window_error gives their error.  Every generic leaf mode is covered.
 * Render-temporal assets (profile 1): frames [t0, t0 + n), n <= 64, d_out[f * frame_stride +
 * rank * 512 + voxel] over the active leaves of the current page table (vbt_build_page_table
 * first), as vbt_decode_cache, in consecutive windows of 16 frames.  Per leaf and window, the
 * union U of all controls' key frames inside the window plus its first and last frame are the
 * knots; between knots every voxel is linear in t
 * (decodeFromSequence, src/render_temporal_decode.cpp:79-131, is piecewise linear in t and the
 * trilinear is linear in the controls).  The voxels at the K = |U| knots are decoded exactly on
 * the CUDA cores and the window is V(512 x n) = Coef(512 x K) . H(K x n) on tcgen05 tensor cores,
 * H the hat functions of U, both split into three BF16 terms, FP32 accumulation.  Knot frames are
 * bit-identical to vbt_decode_cache; Mode2 leaves and leaves whose keys do not strictly increase
 * take every frame as a knot, and a window whose every frame is a knot is decoded exactly without
 * the contraction.  d_out 16-byte aligned, frame_stride a multiple of 4. */
int vbt_decode_window(vbt_asset* asset, int t0, int n, float* d_out, uint64_t frame_stride, void* stream);
/* FP64 error oracle on the GPU for any cache of frames [t0, t0 + n) (from vbt_decode_window or
 * vbt_decode_cache; render assets: the active ranks of the current page table): the reference
 * model evaluated in double without intermediate rounding (same FP32 coefficients, basis values,
 * key values and trilinear weights; the bracket the reference's key search selects) and reduced in
 * double.  stats[0] = max |value - oracle|, stats[1] = rms, stats[2] / stats[3] = oracle min / max.
 * Synchronises `stream`. */
int vbt_window_error(vbt_asset* asset, int t0, int n, const float* d_values, uint64_t frame_stride, double* stats,
                     void* stream);

/* Self-test, no counterpart in the reference.  The render decode forms the interpolation weight
 * (t - f0) / (f1 - f0) of src/render_temporal_decode.cpp:129-130 without a division: one
 * reciprocal per key interval and a Markstein correction per frame.  This compares that quotient
 * with IEEE division on `device` for every integer pair 0 < a < b <= b_max (b_max <= 65535, the
 * widest key-frame span).  result[0] = mismatches, result[1] = smallest failing (b << 16 | a), or
 * all ones when there is none.  Synchronous. */
int vbt_selftest_key_division(uint32_t b_max, uint64_t* result, int device);

/* ---- Batched timeline: autotuned, graph-captured ---------------------------------------------
 * No counterpart in the reference.  The current-frame cache of a frame range is a page-table build
 * plus one decode launch per `frames_per_launch` frames.  The launch shape (leaf per CTA: the
 * TMA-staged kernel; leaf per warp: eight leaves per CTA), the frames per launch and the grid are
 * chosen per asset by timing the candidates on the caller's output (vbt_autotune_cache), or set
 * directly (vbt_set_tuning).  vbt_decode_cache_timeline then runs the whole range; with use_graph
 * it is captured once into a CUDA graph per (first frame, count, output, stride) and replayed with
 * one cudaGraphLaunch.  Output as vbt_decode_cache: d_out[f * frame_stride + rank * 512 + voxel]. */
typedef struct {
    uint32_t variant;            /* 0: leaf per CTA; 1: leaf per warp */
    uint32_t frames_per_launch;  /* 1 .. 64 */
    int grid;                    /* CTAs per launch, 0 = one wave */
    float ms_per_frame;          /* measured by vbt_autotune_cache (0 when set by hand) */
    float ms_per_frame_default;  /* the untuned configuration (leaf per CTA, 48 frames, one wave) */
} vbt_tuning;

/* Times every candidate over frames [0, nframes) into d_out (frame_stride floats per frame),
 * keeps the fastest for the asset and returns it.  Synchronises `stream`. */
int vbt_autotune_cache(vbt_asset* asset, int nframes, float* d_out, uint64_t frame_stride, vbt_tuning* out,
                       void* stream);
int vbt_set_tuning(vbt_asset* asset, const vbt_tuning* tuning);
int vbt_get_tuning(vbt_asset* asset, vbt_tuning* out);
/* Page table + cache of frames [t0, t0 + n) with the asset's tuning.  The first call with
 * use_graph for a given (t0, n, d_out, frame_stride) captures the graph on `stream` (which must not
 * be the legacy default stream); a graph is never replayed concurrently with itself, and changing
 * the tuning drops the captured graphs. */
int vbt_decode_cache_timeline(vbt_asset* asset, int t0, int n, float* d_out, uint64_t frame_stride, int use_graph,
                              void* stream);

/* ---- Serving loop -----------------------------------------------------------------------------
 * No counterpart in the reference (its decoders are one call per value or per frame).  A server
 * keeps several resident assets, accepts point, slice and frame requests from any thread, admits
 * them while an HBM budget for their inputs and results has room, and runs the requests admitted
 * together -- points, slices and frames of any assets, mixed -- as one persistent launch whose
 * warps take tiles of all of them from a work counter (a CUDA graph per stream, its parameters
 * updated each step).  Launches run on `slots` streams, so that requests arriving while others are
 * on the GPU overlap with them (continuous batching).  One scheduler thread per server issues all
 * GPU work.  Results are identical to the one-asset calls above (tested alone versus in a mix). */
typedef struct vbt_server vbt_server;

typedef struct {
    int device;                  /* CUDA device of the server and of every asset added to it */
    uint64_t hbm_budget_bytes;   /* device memory for in-flight inputs and not yet released results */
    uint64_t host_staging_bytes; /* pinned host memory for requests with pageable host buffers */
    uint32_t slots;              /* launch streams, 1 .. 32 (units in flight at once) */
    uint32_t max_batch_queries;  /* values (points, slice and frame voxels) merged into one launch,
                                  * 0 = 4,194,304; a larger request runs alone */
    uint32_t plain;              /* 1: one request per launch, one launch in flight, FIFO, each kind
                                  * on its own kernel (the baseline) */
    uint32_t separate_kinds;     /* 1: merge only point requests (one multi-asset point launch);
                                  * slices and frames each on their own kernel */
} vbt_server_config;

#define VBT_REQ_POINTS 1u   /* points[n_points] = (x, y, z, t) quads -> n_points floats */
#define VBT_REQ_SLICE 2u    /* z layer over frames [t0, t1) -> (t1 - t0) * X * Y floats */
#define VBT_REQ_FRAMES 3u   /* frames[n_frames] -> n_frames * X * Y * Z floats (dense, clamped) */

typedef struct {
    uint32_t kind;               /* VBT_REQ_* */
    uint32_t asset;              /* id returned by vbt_server_add_asset */
    const uint32_t* points;      /* POINTS: host array (pageable or pinned) or device memory (a
                                  * client that keeps its query batches on the GPU); must stay valid
                                  * until the request is done */
    uint64_t n_points;
    uint32_t z;                  /* SLICE */
    int32_t t0, t1;
    const int32_t* frames;       /* FRAMES: host array (copied at submit) */
    uint32_t n_frames;
    float* host_out;             /* result destination (host memory, pinned or pageable, or device
                                  * memory), or NULL to keep the result in the server's device
                                  * memory until vbt_serve_release */
} vbt_request;

typedef struct {
    int status;                  /* VBT_STATUS_* of the request (decode errors included) */
    uint32_t bad_leaf;           /* first failing leaf when status is a decode status */
    uint64_t result_floats;
    const float* device_result;  /* when host_out was NULL: the result, valid until release */
    double submit_ms, start_ms, done_ms;   /* server clock: submitted, launched, seen complete */
} vbt_request_result;

typedef struct {
    uint64_t requests_done, points_done, voxels_done;   /* voxels: slice and frame outputs */
    uint64_t launches, units;          /* kernel launches; launch groups */
    uint64_t arena_peak_bytes, arena_bytes, resident_asset_bytes;
    double p50_ms, p99_ms, max_ms;     /* submit -> done, over requests done since the last reset */
    double busy_ms;                    /* wall time with at least one unit in flight */
} vbt_server_stats;

int vbt_server_create(const vbt_server_config* config, vbt_server** out);
/* The asset stays owned by the caller and must outlive the server; at most 64 assets, all on the
 * server's device. */
int vbt_server_add_asset(vbt_server* server, vbt_asset* asset, uint32_t* asset_id);
/* VBT_STATUS_LIMIT when the request alone needs more than the budget. */
int vbt_serve_submit(vbt_server* server, const vbt_request* request, uint64_t* ticket);
int vbt_serve_poll(vbt_server* server, uint64_t ticket, int* done, vbt_request_result* result);
int vbt_serve_wait(vbt_server* server, uint64_t ticket, vbt_request_result* result);
/* Frees the ticket and a device-resident result; every ticket must be released once done. */
int vbt_serve_release(vbt_server* server, uint64_t ticket);
int vbt_server_get_stats(vbt_server* server, vbt_server_stats* out);
int vbt_server_reset_stats(vbt_server* server);
/* Waits for all submitted requests, then frees the server's streams and memory. */
int vbt_server_destroy(vbt_server* server);

#ifdef __cplusplus
}
#endif
#endif
