/*
 * vbt_oracle.h -- CPU restatement of VBT's compressed-domain temporal decode path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * path in vbt_b200/.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it; the product never links or calls it.
 *
 * Every function restates one function of the reference (VBT, namespace vbt /
 * vbt::render) and cites the file:line it follows.  The restatement is pinned
 * against (1) the known-answer cases of the reference's own tests
 * (tests/temporal_decode_tests.cpp, tests/render_temporal_payload_tests.cpp,
 * tests/vbt_file_tests.cpp), rebuilt as fixtures under tests/golden/, and
 * (2) the reference decoder itself, compiled from its sources into
 * oracle/_ref/ by oracle/Makefile and compared on every asset the tests use.
 */
#ifndef VBT_ORACLE_H
#define VBT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: identical numbering to include/vbt_b200.h (VBT_STATUS_*). */
enum {
    VO_OK = 0,
    VO_ERR_LEAF_TOO_SMALL = 1,
    VO_ERR_PREFIX_MISSING = 2,
    VO_ERR_LEAF_SHORT = 3,
    VO_ERR_SHELL_OCC_OOB = 4,
    VO_ERR_SHELL_GROUP_PREFIX = 5,
    VO_ERR_SHELL_NO_ACTIVE = 6,
    VO_ERR_SHELL_RESIDUAL_OOB = 7,
    VO_ERR_SHELL_TRAILING = 8,
    VO_ERR_CONTROL_INDEX = 9,
    VO_ERR_STREAM_OOB = 10,
    VO_ERR_DECODE_OOB = 11,
    VO_ERR_KEY_RANGE_OOB = 12,
    VO_ERR_KEY_INDEX = 13,
};

typedef struct {
    uint32_t mode, coarse_codec, fine_codec, coarse_res, fine_res;
} vo_header;

typedef struct {
    uint32_t desc_off, desc_bytes, bin_off, bin_bytes, key_off, key_bytes, total;
} vo_stream_layout;

typedef struct {
    vo_header header;
    uint32_t coarse_kf, fine_kf;
    uint32_t coarse_off, fine_off, total;
    vo_stream_layout coarse, fine;
    uint32_t shell_active, shell_residual_off, shell_residual_bytes;
} vo_leaf_view;

/* VBTPACK4 file as loaded by render/src/vbt_file.cpp:109-210. */
typedef struct {
    uint32_t version, width, height, depth, frames, leaf_size, coarse_res, max_coarse_keep,
        leaf_count, profile_type, scale_count;
    float* scales;
    uint32_t* offsets;      /* leaf_count + 1 words */
    uint32_t* payload;      /* offsets[leaf_count] words */
    uint64_t payload_words;
} vo_file;

uint32_t vo_pack_header(const vo_header* h);
void vo_unpack_header(uint32_t packed, vo_header* out);
void vo_leaf_layout(const vo_header* h, uint32_t coarse_kf, uint32_t fine_kf, int align4, vo_leaf_view* out);
int vo_parse_leaf(const uint8_t* leaf, size_t bytes, int align4, vo_leaf_view* out);
float vo_half_to_float(uint16_t bits);
uint16_t vo_float_to_half(float v);

int vo_decode_control(const uint8_t* stream, uint32_t codec, uint32_t control_count, uint32_t bins,
                      uint32_t kf_count, uint32_t stream_bytes, int align4, int total_frames,
                      uint32_t control_index, int frame, float* out);
int vo_decode_shell_voxel(const uint8_t* leaf, const vo_leaf_view* v, int total_frames,
                          uint32_t voxel, int frame, float* out);
int vo_decode_leaf_frame(const uint8_t* leaf, size_t bytes, int total_frames, int frame,
                         int w, int h, int d, float* out);

int vo_load_file(const char* path, vo_file* out, char* err, size_t err_len);
int vo_load_image(const uint8_t* bytes, uint64_t len, vo_file* out, char* err, size_t err_len);
void vo_free_file(vo_file* f);

/* Render-temporal family (profileType 0/1). */
int vo_decode_frame(const vo_file* f, int frame, float* out, int threads, uint32_t* bad_leaf);
uint32_t vo_build_page_table(const vo_file* f, uint32_t* compact);
int vo_decode_cache(const vo_file* f, int frame, const uint32_t* compact, float* cache, int threads);
int vo_query_points(const vo_file* f, const uint32_t* xyzt, uint64_t n, float* out, int threads);

/* Scientific family (profileType 2). */
float vo_sci_value(const vo_file* f, uint32_t x, uint32_t y, uint32_t z, uint32_t t);
void vo_sci_frame(const vo_file* f, uint32_t frame, float* out, int threads);
void vo_sci_query_points(const vo_file* f, const uint32_t* xyzt, uint64_t n, float* out, int threads);
double vo_dct_basis_f64(int total, int index, int k);
float vo_dct_basis(int total, int index, int k);

/* The Studio's control cache and ray sampler (vbt_sample_oracle.c): the push constants of
 * VBTStudio/frontend/shaders/vbt_sample.comp:38-66 that are not the asset's own geometry.
 * up_axis is the shader's `padding` field (2: z up for the floor plane and key light). */
typedef struct {
    uint32_t step_count;
    int32_t frame_index;
    float bbox_min[3];
    uint32_t render_mode;      /* 0 density accumulation, 1 level-set surface */
    float voxel_size, background_value, surface_iso, surface_epsilon_voxels, surface_normal_step, max_step_voxels;
    uint32_t surface_model;
    float floor_height;
    uint32_t shadow_steps;
    uint32_t up_axis;
} vo_sample_params;
int vo_control_cache(const vo_file* f, int frame, const uint32_t* compact, float* cache576);
void vo_sample_rays(const vo_file* f, const float* cache576, const uint32_t* compact, const vo_sample_params* p,
                    const float* rays, uint32_t n, float* results);
/* render/shaders/vbt_smoke_sample.comp over the payload (step_count, frame_index, bbox_min of p). */
void vo_smoke_sample_rays(const vo_file* f, const vo_sample_params* p, const float* rays, uint32_t n, float* out);

/* The encoder's per-voxel keyframe pass (vbt_keyframe_oracle.c): DensityTemporalProfile of
 * src/render_temporal_kf_probe_main.cpp:81-95 plus the background threshold of :477 (< 0: off). */
typedef struct {
    float eps_abs, eps_rel, gamma_delta, render_cutoff, cutoff_band;
    uint32_t cutoff_temporal_protect, iso_surface_protect;
    float iso_value, iso_band;
    double bg_threshold;
} vo_keyframe_profile;
int vo_detect_keyframes(const float* values, int n, const vo_keyframe_profile* p, int* keys, int* used_protect);
void vo_reconstruct(const float* values, int n, const int* keys, int key_count, float* out);
void vo_keyframe_pass(const float* values, uint64_t series, int frames, uint64_t frame_stride,
                      const vo_keyframe_profile* p, uint32_t* key_mask, uint32_t* key_count, uint8_t* flags,
                      float* recon, double* err2, int threads);
int vo_coarse_fit(const float* leaf_recon, int frames, int w, int h, int d, const vo_keyframe_profile* control_profile,
                  uint32_t* desc, uint8_t* bins, uint16_t* key_frames, float* key_values, int key_cap,
                  int* required_max_local, float* grid);
void vo_float_to_half_n(const float* v, uint64_t n, uint16_t* out);
int vo_shell_fit(const float* leaf_recon, int frames, int w, int h, int d, const vo_keyframe_profile* control_profile,
                 const float* coarse_grid, int levelset, float surface_band, float guard_band, float temporal_band,
                 float shell_cut, uint8_t* occupancy80, uint32_t* desc, uint8_t* bins, uint16_t* key_frames,
                 float* key_values, int key_cap, int* active_count, int* required_max_local);
int vo_fine6_fit(const float* leaf_recon, int frames, int w, int h, int d, const vo_keyframe_profile* control_profile,
                 const float* coarse_grid, uint32_t* desc, uint8_t* bins, uint16_t* key_frames, float* key_values,
                 int key_cap, int* required_max_local, float* grid);

#ifdef __cplusplus
}
#endif
#endif
