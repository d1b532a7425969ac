/*
 * vbt_oracle.c -- CPU restatement of VBT's compressed-domain temporal decode.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker; see vbt_oracle.h).  Plain C11,
 * built with -ffp-contract=off so every float operation rounds exactly where
 * the reference's does (the reference is compiled for baseline x86-64, which
 * has no FMA).  All file:line citations are paths inside the VBT project.
 */
#define _POSIX_C_SOURCE 200809L /* fmemopen */
#include "vbt_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MODE_EMPTY 0u
#define MODE_GRID4 1u
#define MODE_FINE_COMPACT 2u
#define MODE_FINE6 3u

static uint32_t align4(uint32_t b) { return (b + 3u) & ~3u; }
static uint32_t rd_u16(const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8); }
static uint32_t rd_u32(const uint8_t* p)
{
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static uint64_t rd_u64(const uint8_t* p) { return (uint64_t)rd_u32(p) | ((uint64_t)rd_u32(p + 4) << 32); }
static int popcount64(uint64_t w)
{
    int c = 0;
    for (; w; w &= w - 1u) ++c;
    return c;
}

/* src/render_temporal_payload.cpp:30-40 renderTemporalKeyframeBytes: 8 for FP32 (codec 1), 3 otherwise. */
static uint32_t key_stride(uint32_t codec) { return codec == 1u ? 8u : 3u; }

/* src/render_temporal_payload.cpp:87-96 packRenderTemporalHeader */
uint32_t vo_pack_header(const vo_header* h)
{
    uint32_t p = 0;
    p |= h->mode & 3u;
    p |= (h->coarse_codec & 3u) << 2;
    p |= (h->fine_codec & 3u) << 4;
    p |= ((h->coarse_res < 7u ? h->coarse_res : 7u) & 7u) << 6;
    p |= ((h->fine_res < 7u ? h->fine_res : 7u) & 7u) << 9;
    return p;
}

/* src/render_temporal_payload.cpp:98-107 unpackRenderTemporalHeader */
void vo_unpack_header(uint32_t packed, vo_header* out)
{
    out->mode = packed & 3u;
    out->coarse_codec = (packed >> 2) & 3u;
    out->fine_codec = (packed >> 4) & 3u;
    out->coarse_res = (packed >> 6) & 7u;
    out->fine_res = (packed >> 9) & 7u;
}

/* src/render_temporal_payload.cpp:62-78 computeStreamLayout */
static void stream_layout(uint32_t start, uint32_t controls, uint32_t bins, uint32_t kf, uint32_t codec,
                          int align, vo_stream_layout* s)
{
    s->desc_off = start;
    s->desc_bytes = controls * 4u;
    s->bin_off = s->desc_off + s->desc_bytes;
    s->bin_bytes = align ? align4(controls * bins) : controls * bins;
    s->key_off = s->bin_off + s->bin_bytes;
    s->key_bytes = align ? align4(kf * key_stride(codec)) : kf * key_stride(codec);
    s->total = s->desc_bytes + s->bin_bytes + s->key_bytes;
}

/* src/render_temporal_payload.cpp:143-197 computeRenderTemporalLeafLayout */
void vo_leaf_layout(const vo_header* h, uint32_t coarse_kf, uint32_t fine_kf, int align, vo_leaf_view* v)
{
    memset(&v->coarse, 0, sizeof v->coarse);
    memset(&v->fine, 0, sizeof v->fine);
    v->coarse_off = 8u;
    const uint32_t cc = h->coarse_res * h->coarse_res * h->coarse_res;
    const uint32_t fc = h->fine_res * h->fine_res * h->fine_res;
    stream_layout(v->coarse_off, cc, 8u, coarse_kf, h->coarse_codec, align, &v->coarse);
    v->fine_off = v->coarse_off + v->coarse.total;
    if (h->mode == MODE_FINE6) {
        stream_layout(v->fine_off, fc, 8u, fine_kf, h->fine_codec, align, &v->fine);
        v->total = v->fine_off + v->fine.total;
    } else if (h->mode == MODE_FINE_COMPACT) {
        v->fine.desc_off = v->fine_off;
        v->fine.desc_bytes = 80u;
        v->fine.bin_off = v->fine_off + 80u;
        v->fine.bin_bytes = 0u;
        v->fine.key_off = v->fine_off + 80u;
        v->fine.key_bytes = align ? align4(fine_kf * key_stride(h->fine_codec)) : fine_kf * key_stride(h->fine_codec);
        v->fine.total = 80u + v->fine.key_bytes;
        v->total = v->fine_off + v->fine.total;
    } else {
        v->total = v->coarse_off + v->coarse.total;
    }
    if (h->mode == MODE_EMPTY) {
        v->coarse_off = 0;
        v->fine_off = 0;
        memset(&v->coarse, 0, sizeof v->coarse);
        memset(&v->fine, 0, sizeof v->fine);
        v->total = 4u;
    }
}

/* src/render_temporal_payload.cpp:234-311 parseRenderTemporalPackedLeaf */
int vo_parse_leaf(const uint8_t* leaf, size_t bytes, int align, vo_leaf_view* v)
{
    memset(v, 0, sizeof *v);
    if (leaf == NULL || bytes < 4u) return VO_ERR_LEAF_TOO_SMALL;
    vo_unpack_header(rd_u32(leaf), &v->header);
    if (v->header.mode == MODE_EMPTY) {
        vo_leaf_layout(&v->header, 0, 0, align, v);
        return VO_OK;
    }
    if (bytes < 8u) return VO_ERR_PREFIX_MISSING;
    v->coarse_kf = rd_u16(leaf + 4);
    v->fine_kf = rd_u16(leaf + 6);
    vo_leaf_layout(&v->header, v->coarse_kf, v->fine_kf, align, v);
    if (v->total > bytes) return VO_ERR_LEAF_SHORT;
    if (v->header.mode == MODE_FINE_COMPACT) {
        const size_t occ_off = v->fine.desc_off;
        const size_t occ_bytes = v->fine.desc_bytes;
        if (occ_bytes != 80u || occ_off > bytes || occ_bytes > bytes - occ_off) return VO_ERR_SHELL_OCC_OOB;
        uint32_t expect = 0; /* uint16 in the reference; <= 512 here */
        for (int g = 0; g < 8; ++g) {
            if (rd_u16(leaf + occ_off + 64 + 2 * g) != (expect & 0xFFFFu)) return VO_ERR_SHELL_GROUP_PREFIX;
            expect += (uint32_t)popcount64(rd_u64(leaf + occ_off + 8 * g));
        }
        if (expect == 0u) return VO_ERR_SHELL_NO_ACTIVE;
        size_t res_off = occ_off + occ_bytes;
        if (align) res_off = (res_off + 3u) & ~(size_t)3u;
        const size_t desc = (size_t)expect * 4u;
        size_t binb = (size_t)expect * 4u;
        size_t keyb = (size_t)v->fine_kf * key_stride(v->header.fine_codec);
        if (align) {
            binb = (binb + 3u) & ~(size_t)3u;
            keyb = (keyb + 3u) & ~(size_t)3u;
        }
        const size_t res_bytes = desc + binb + keyb;
        if (res_off > bytes || res_bytes > bytes - res_off) return VO_ERR_SHELL_RESIDUAL_OOB;
        if (res_off + res_bytes != bytes) return VO_ERR_SHELL_TRAILING;
        v->shell_active = expect;
        v->shell_residual_off = (uint32_t)res_off;
        v->shell_residual_bytes = (uint32_t)res_bytes;
    }
    return VO_OK;
}

/* src/render_temporal_decode.cpp:167-199 renderTemporalHalfBitsToFloat */
float vo_half_to_float(uint16_t bits)
{
    const uint32_t sign = ((uint32_t)(bits & 0x8000u)) << 16;
    uint32_t e = (bits >> 10) & 0x1Fu, m = bits & 0x3FFu, out;
    if (e == 0) {
        if (m == 0) {
            out = sign;
        } else {
            e = 1;
            while ((m & 0x400u) == 0) {
                m <<= 1;
                --e;
            }
            m &= 0x3FFu;
            out = sign | ((e + 127u - 15u) << 23) | (m << 13);
        }
    } else if (e == 31) {
        out = sign | 0x7F800000u | (m << 13);
    } else {
        out = sign | ((e + 127u - 15u) << 23) | (m << 13);
    }
    float f;
    memcpy(&f, &out, 4);
    return f;
}

/* src/render_temporal_decode.cpp:133-165 renderTemporalFloatToHalfBits */
uint16_t vo_float_to_half(float value)
{
    uint32_t bits;
    memcpy(&bits, &value, 4);
    const uint32_t sign = (bits >> 16) & 0x8000u;
    int32_t e = (int32_t)((bits >> 23) & 0xFFu) - 127 + 15;
    uint32_t m = bits & 0x7FFFFFu;
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        m |= 0x800000u;
        const uint32_t shifted = m >> (uint32_t)(1 - e);
        return (uint16_t)(sign | ((shifted + 0x1000u) >> 13));
    }
    if (e >= 31) return (uint16_t)(sign | 0x7C00u);
    const uint32_t rm = (m + 0x1000u) >> 13;
    if (rm == 0x400u) {
        e += 1;
        if (e >= 31) return (uint16_t)(sign | 0x7C00u);
        return (uint16_t)(sign | ((uint32_t)e << 10));
    }
    return (uint16_t)(sign | ((uint32_t)e << 10) | (rm & 0x3FFu));
}

/* src/render_temporal_decode.cpp:68-77 readPackedKeyframeFrame (unchecked, as in the reference) */
static int key_frame(const uint8_t* kb, uint32_t codec, uint32_t i)
{
    const size_t o = (size_t)i * key_stride(codec);
    return codec == 1u ? (int)rd_u16(kb + o) : (int)kb[o];
}

/* src/render_temporal_decode.cpp:33-66 readPackedKeyframe (value part, bounds-checked) */
static int key_value(const uint8_t* kb, uint32_t codec, uint32_t i, uint32_t kf, float* out)
{
    if (i >= kf) return VO_ERR_KEY_INDEX;
    const size_t o = (size_t)i * key_stride(codec);
    const size_t limit = (size_t)kf * key_stride(codec);
    if (codec == 1u) {
        if (o + 8u > limit) return VO_ERR_DECODE_OOB;
        uint32_t b = rd_u32(kb + o + 4);
        memcpy(out, &b, 4);
    } else {
        if (o + 3u > limit) return VO_ERR_DECODE_OOB;
        *out = vo_half_to_float((uint16_t)(kb[o + 1] | (kb[o + 2] << 8)));
    }
    return VO_OK;
}

/* src/render_temporal_decode.cpp:79-131 decodeFromSequence */
static int decode_sequence(const uint8_t* kb, uint32_t codec, uint32_t kf, uint32_t ks, uint32_t kc,
                           const uint8_t* lbin, uint32_t bins, int total, int frame_index, float* out)
{
    if (kc == 0) {
        *out = 0.0f;
        return VO_OK;
    }
    const int tmax = total - 1 > 0 ? total - 1 : 0;
    const int frame = frame_index < 0 ? 0 : (frame_index > tmax ? tmax : frame_index);
    const uint32_t last = kc - 1u;
    uint32_t bin = 0;
    if (bins != 0) {
        const uint32_t q = (uint32_t)(((int64_t)frame * bins) / (total > 1 ? total : 1));
        bin = q < bins - 1u ? q : bins - 1u;
    }
    uint32_t lo = bins == 0 ? 0u : (lbin[bin] < last ? lbin[bin] : last);
    int f0 = key_frame(kb, codec, ks + lo);
    if (f0 > frame) {
        lo = 0u;
        f0 = key_frame(kb, codec, ks);
    }
    if (f0 >= frame || lo == last) return key_value(kb, codec, ks + lo, kf, out);
    uint32_t hi = last;
    if (bin + 1u < bins) {
        const uint32_t h = (uint32_t)lbin[bin + 1u] + 1u;
        hi = h < last ? h : last;
    }
    if (hi < lo + 1u) hi = lo + 1u;
    int f1 = key_frame(kb, codec, ks + hi);
    if (f1 < frame) {
        hi = last;
        f1 = key_frame(kb, codec, ks + hi);
    }
    if (f1 <= frame) return key_value(kb, codec, ks + hi, kf, out);
    while (hi > lo + 1u) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        const int fm = key_frame(kb, codec, ks + mid);
        if (fm < frame) {
            lo = mid;
            f0 = fm;
        } else {
            hi = mid;
            f1 = fm;
        }
    }
    float v1, v0;
    int st = key_value(kb, codec, ks + hi, kf, &v1);
    if (st) return st;
    if (f1 == frame) {
        *out = v1;
        return VO_OK;
    }
    st = key_value(kb, codec, ks + lo, kf, &v0);
    if (st) return st;
    const float alpha = (float)(frame - f0) / (float)(f1 - f0);
    const float diff = v1 - v0;
    const float step = alpha * diff;
    *out = v0 + step;
    return VO_OK;
}

/* src/render_temporal_decode.cpp:304-356 decodeRenderTemporalControlValue */
int vo_decode_control(const uint8_t* s, uint32_t codec, uint32_t cc, uint32_t bins, uint32_t kf,
                      uint32_t stream_bytes, int align, int total, uint32_t ci, int frame, float* out)
{
    if (ci >= cc) return VO_ERR_CONTROL_INDEX;
    const uint32_t descb = cc * 4u;
    uint32_t binb = cc * bins;
    uint32_t keyb = kf * key_stride(codec);
    if (align) {
        binb = align4(binb);
        keyb = align4(keyb);
    }
    if (descb + binb + keyb > stream_bytes) return VO_ERR_STREAM_OOB;
    if ((size_t)ci * 4u + 4u > stream_bytes) return VO_ERR_DECODE_OOB;
    const uint32_t ks = rd_u16(s + (size_t)ci * 4u);
    const uint32_t kc = s[(size_t)ci * 4u + 2u];
    if (kc == 0) {
        *out = 0.0f;
        return VO_OK;
    }
    if (ks + kc > kf) return VO_ERR_KEY_RANGE_OOB;
    return decode_sequence(s + descb + binb, codec, kf, ks, kc, s + descb + (size_t)ci * bins, bins, total, frame, out);
}

/* src/render_temporal_decode.cpp:404-450 decodeRenderTemporalLeafShellVoxelValue */
int vo_decode_shell_voxel(const uint8_t* leaf, const vo_leaf_view* v, int total, uint32_t voxel, int frame,
                          float* out)
{
    *out = 0.0f;
    if (leaf == NULL || voxel >= 512u) return VO_OK;
    if (v->header.mode != MODE_FINE_COMPACT) return VO_OK;
    const uint32_t g = voxel >> 6, bit = voxel & 63u;
    if (v->fine.desc_bytes < 80u) return VO_OK; /* unpack of a short section yields zeros */
    const uint8_t* occ = leaf + v->fine.desc_off;
    const uint64_t mask = rd_u64(occ + 8 * g);
    if ((mask & (1ull << bit)) == 0ull) return VO_OK;
    const uint32_t di = (rd_u16(occ + 64 + 2 * g) + (uint32_t)popcount64(mask & ((1ull << bit) - 1ull))) & 0xFFFFu;
    if (v->shell_active == 0 || v->fine_kf == 0) return VO_OK;
    return vo_decode_control(leaf + v->shell_residual_off, v->header.fine_codec, v->shell_active, 4u, v->fine_kf,
                             v->shell_residual_bytes, 1, total, di, frame, out);
}

/* render/src/render_smoke_vbt_bench_main.cpp:201-249 controlCoords + locateCoord.
 * Resolutions 0 and 1 index past the end of the coordinate vector in the reference (undefined
 * behaviour); here resolution 1 yields the single control and resolution 0 yields 0. */
static void locate(float p, int extent, int res, int* i0, int* i1, float* w)
{
    const float scale = 7.0f / (float)(res - 1);
    const float maxp = (float)(extent - 1 > 0 ? extent - 1 : 0);
    p = p < 0.0f ? 0.0f : (p > maxp ? maxp : p);
    int j1 = 1;
    while (j1 < res - 1 && (float)j1 * scale < p) ++j1;
    const int j0 = j1 - 1 > 0 ? j1 - 1 : 0;
    const float c0 = (float)j0 * scale, c1 = (float)j1 * scale;
    *i0 = j0;
    *i1 = j1;
    *w = (c1 > c0) ? ((p - c0) / (c1 - c0)) : 0.0f;
}

static float lerp_w(float a, float b, float t)
{
    const float omt = 1.0f - t;
    const float x = a * omt;
    const float y = b * t;
    return x + y;
}

/* render/src/render_smoke_vbt_bench_main.cpp:236-267 sampleControlGrid */
static float sample_grid(const float* g, int res, int w, int h, int d, int lx, int ly, int lz)
{
    if (res <= 0) return 0.0f;
    if (res == 1) return g[0];
    int x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
    locate((float)lx, w, res, &x0, &x1, &tx);
    locate((float)ly, h, res, &y0, &y1, &ty);
    locate((float)lz, d, res, &z0, &z1, &tz);
#define AT(ix, iy, iz) g[((iz) * res + (iy)) * res + (ix)]
    const float c00 = lerp_w(AT(x0, y0, z0), AT(x1, y0, z0), tx);
    const float c01 = lerp_w(AT(x0, y0, z1), AT(x1, y0, z1), tx);
    const float c10 = lerp_w(AT(x0, y1, z0), AT(x1, y1, z0), tx);
    const float c11 = lerp_w(AT(x0, y1, z1), AT(x1, y1, z1), tx);
#undef AT
    const float c0 = lerp_w(c00, c10, ty);
    const float c1 = lerp_w(c01, c11, ty);
    return lerp_w(c0, c1, tz);
}

/* render/src/render_smoke_vbt_bench_main.cpp:277-387 decodeLeafFrameValues.
 * out[] is indexed (lz*h + ly)*w + lx over the cropped extent, as in the reference. */
int vo_decode_leaf_frame(const uint8_t* leaf, size_t bytes, int total, int frame, int w, int h, int d, float* out)
{
    vo_leaf_view v;
    int st = vo_parse_leaf(leaf, bytes, 1, &v);
    if (st) return st;
    const int n = w * h * d;
    if (v.header.mode == MODE_EMPTY) {
        for (int i = 0; i < n; ++i) out[i] = 0.0f;
        return VO_OK;
    }
    const int cres = (int)v.header.coarse_res, fres = (int)v.header.fine_res;
    const uint32_t cc = (uint32_t)(cres * cres * cres);
    float coarse[343], fine[343];
    for (uint32_t i = 0; i < cc; ++i) {
        st = vo_decode_control(leaf + v.coarse_off, v.header.coarse_codec, cc, 8u, v.coarse_kf, v.coarse.total, 1,
                               total, i, frame, &coarse[i]);
        if (st) return st;
    }
    const int has_fine = fres > 0 && v.fine.total > 0 && v.header.mode != MODE_GRID4;
    uint32_t fc = 0;
    if (has_fine) {
        fc = (uint32_t)(fres * fres * fres);
        for (uint32_t i = 0; i < fc; ++i) {
            st = vo_decode_control(leaf + v.fine_off, v.header.fine_codec, fc, 8u, v.fine_kf, v.fine.total, 1, total,
                                   i, frame, &fine[i]);
            if (st) return st;
        }
    }
    const int has_occ = v.header.mode == MODE_FINE_COMPACT;
    const uint8_t* occ = has_occ ? leaf + v.fine.desc_off : NULL;
    for (int lz = 0; lz < d; ++lz)
        for (int ly = 0; ly < h; ++ly)
            for (int lx = 0; lx < w; ++lx) {
                const uint32_t vox = (uint32_t)((lz * 8 + ly) * 8 + lx);
                float value = sample_grid(coarse, cres, w, h, d, lx, ly, lz);
                if (fc > 0) {
                    value = value + sample_grid(fine, fres, w, h, d, lx, ly, lz);
                } else if (v.header.mode == MODE_FINE_COMPACT) {
                    float r;
                    st = vo_decode_shell_voxel(leaf, &v, total, vox, frame, &r);
                    if (st) return st;
                    value = value + r;
                }
                if (has_occ && ((rd_u64(occ + 8 * (vox >> 6)) >> (vox & 63u)) & 1ull) == 0ull && value < 0.0f)
                    value = 0.0f;
                out[(lz * h + ly) * w + lx] = value;
            }
    return VO_OK;
}

/* ---------------- VBTPACK4 reader: render/src/vbt_file.cpp:39-210 ---------------- */

static void set_err(char* err, size_t n, const char* msg)
{
    if (err && n) snprintf(err, n, "%s", msg);
}

static int load_stream(FILE* fp, vo_file* out, char* err, size_t n);

int vo_load_file(const char* path, vo_file* out, char* err, size_t n)
{
    memset(out, 0, sizeof *out);
    FILE* fp = fopen(path, "rb");
    if (!fp) {
        char b[512];
        snprintf(b, sizeof b, "Failed to query file size: %s", path);
        set_err(err, n, b);
        return -1;
    }
    return load_stream(fp, out, err, n);
}

/* The same checks and copies over a file image held in memory (read through fmemopen). */
int vo_load_image(const uint8_t* bytes, uint64_t len, vo_file* out, char* err, size_t n)
{
    memset(out, 0, sizeof *out);
    FILE* fp = (bytes && len) ? fmemopen((void*)bytes, (size_t)len, "rb") : NULL;
    if (!fp) {
        set_err(err, n, "Invalid VBTPACK4 file size.");
        return -1;
    }
    return load_stream(fp, out, err, n);
}

static int load_stream(FILE* fp, vo_file* out, char* err, size_t n)
{
    fseek(fp, 0, SEEK_END);
    const uint64_t file_bytes = (uint64_t)ftell(fp);
    fseek(fp, 0, SEEK_SET);
    const uint64_t kHeader = 52u;
    if (file_bytes < kHeader) {
        fclose(fp);
        set_err(err, n, "Invalid VBTPACK4 file size.");
        return -1;
    }
    uint8_t hb[52];
    if (fread(hb, 1, 52, fp) != 52) {
        fclose(fp);
        set_err(err, n, "Failed to read VBTPACK header.");
        return -1;
    }
    uint32_t f[11];
    for (int i = 0; i < 11; ++i) f[i] = rd_u32(hb + 8 + 4 * i);
    out->version = f[0];
    out->width = f[1];
    out->height = f[2];
    out->depth = f[3];
    out->frames = f[4];
    out->leaf_size = f[5];
    out->coarse_res = f[6];
    out->max_coarse_keep = f[7];
    out->leaf_count = f[8];
    out->profile_type = f[9];
    out->scale_count = f[10];
    const char* msg = NULL;
    char vb[96];
    if (memcmp(hb, "VBTPACK4", 8) != 0) msg = "Unsupported magic. Expected VBTPACK4.";
    else if (out->version != 4u) {
        snprintf(vb, sizeof vb, "Unsupported VBTPACK4 version: %u", out->version);
        msg = vb;
    } else if (!out->width || !out->height || !out->depth || !out->frames)
        msg = "VBTPACK4 dimensions and frame count must be non-zero.";
    else if (out->leaf_size != 8u) msg = "VBTPACK4 v4 requires leafSize=8.";
    else if (out->coarse_res == 0u || out->coarse_res > 8u) msg = "Invalid VBTPACK4 coarse resolution.";
    else if (out->profile_type > 2u) msg = "Invalid VBTPACK4 profile type.";
    else if (out->max_coarse_keep > out->frames || out->scale_count > 64u || out->scale_count > out->max_coarse_keep)
        msg = "Invalid VBTPACK4 coarse temporal metadata.";
    if (!msg) {
        const uint64_t lx = ((uint64_t)out->width + 7u) / 8u, ly = ((uint64_t)out->height + 7u) / 8u,
                       lz = ((uint64_t)out->depth + 7u) / 8u;
        const uint64_t expect = lx * ly * lz; /* cannot overflow: each factor < 2^30 */
        if (expect > 0xFFFFFFFFull) msg = "VBTPACK4 leaf count overflows the v4 header.";
        else if (out->leaf_count != expect) msg = "VBTPACK4 leafCount does not match dimensions and leafSize.";
        else if (kHeader + 4ull * out->scale_count + 4ull * ((uint64_t)out->leaf_count + 1u) > file_bytes)
            msg = "VBTPACK4 file is truncated before its offset table.";
    }
    if (msg) {
        fclose(fp);
        set_err(err, n, msg);
        return -1;
    }
    out->scales = (float*)calloc(out->scale_count ? out->scale_count : 1, 4);
    if (out->scale_count && fread(out->scales, 4, out->scale_count, fp) != out->scale_count) {
        fclose(fp);
        vo_free_file(out);
        set_err(err, n, "Failed to read coarse AC scales.");
        return -1;
    }
    out->offsets = (uint32_t*)malloc(4ull * ((uint64_t)out->leaf_count + 1u));
    if (fread(out->offsets, 4, (size_t)out->leaf_count + 1u, fp) != (size_t)out->leaf_count + 1u) {
        fclose(fp);
        vo_free_file(out);
        set_err(err, n, "Failed to read offset table.");
        return -1;
    }
    if (out->offsets[0] != 0u) msg = "VBTPACK4 offset table must begin at word zero.";
    for (uint32_t i = 0; !msg && i < out->leaf_count; ++i)
        if (out->offsets[i] >= out->offsets[i + 1u]) msg = "VBTPACK4 offsets must be strictly increasing for every leaf.";
    if (!msg) {
        const uint64_t words = out->offsets[out->leaf_count];
        const uint64_t expect = kHeader + 4ull * out->scale_count + 4ull * ((uint64_t)out->leaf_count + 1u) + 4ull * words;
        if (expect != file_bytes) msg = expect > file_bytes ? "VBTPACK4 payload is truncated." : "VBTPACK4 file contains trailing bytes.";
        out->payload_words = words;
    }
    if (msg) {
        fclose(fp);
        vo_free_file(out);
        set_err(err, n, msg);
        return -1;
    }
    out->payload = (uint32_t*)malloc(4ull * (out->payload_words ? out->payload_words : 1));
    if (out->payload_words && fread(out->payload, 4, out->payload_words, fp) != out->payload_words) {
        fclose(fp);
        vo_free_file(out);
        set_err(err, n, "Failed to read payload pool.");
        return -1;
    }
    fclose(fp);
    return 0;
}

void vo_free_file(vo_file* f)
{
    free(f->scales);
    free(f->offsets);
    free(f->payload);
    memset(f, 0, sizeof *f);
}

/* ---------------- Render-temporal frame / cache / query composition ---------------- */

static void leaf_geom(const vo_file* f, uint32_t leaf, int* bx, int* by, int* bz, int* w, int* h, int* d)
{
    const uint32_t lx = (f->width + 7u) / 8u, ly = (f->height + 7u) / 8u;
    *bx = (int)(leaf % lx);
    *by = (int)((leaf / lx) % ly);
    *bz = (int)(leaf / (lx * ly));
    const int ex = (int)f->width - *bx * 8, ey = (int)f->height - *by * 8, ez = (int)f->depth - *bz * 8;
    *w = ex < 8 ? ex : 8;
    *h = ey < 8 ? ey : 8;
    *d = ez < 8 ? ez : 8;
}

/* render/src/render_smoke_vbt_bench_main.cpp:389-452 decodeFrameToDense (OpenMP over leaves). */
int vo_decode_frame(const vo_file* f, int frame, float* out, int threads, uint32_t* bad_leaf)
{
    const uint8_t* base = (const uint8_t*)f->payload;
    int status = VO_OK;
    uint32_t bad = 0xFFFFFFFFu;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int64_t li = 0; li < (int64_t)f->leaf_count; ++li) {
        const uint32_t leaf = (uint32_t)li;
        int bx, by, bz, w, h, d;
        leaf_geom(f, leaf, &bx, &by, &bz, &w, &h, &d);
        float vals[512];
        const uint32_t wb = f->offsets[leaf], we = f->offsets[leaf + 1];
        const int st = vo_decode_leaf_frame(base + 4ull * wb, 4ull * (we - wb), (int)f->frames, frame, w, h, d, vals);
        if (st) {
#ifdef _OPENMP
#pragma omp critical
#endif
            {
                if (leaf < bad) {
                    bad = leaf;
                    status = st;
                }
            }
            continue;
        }
        for (int lz = 0; lz < d; ++lz)
            for (int ly = 0; ly < h; ++ly) {
                float* row = out + ((uint64_t)(bz * 8 + lz) * f->height + (uint64_t)(by * 8 + ly)) * f->width + bx * 8;
                memcpy(row, vals + (lz * h + ly) * w, 4u * (uint32_t)w);
            }
    }
    if (bad_leaf) *bad_leaf = bad;
    return status;
}

/* VBTStudio/frontend/shaders/vbt_active_index.comp:28-57: a leaf is active when its header's
 * route tag (bits 0-1) is non-zero; the canonical rank is the ascending exclusive prefix count
 * (the shader's atomic group base makes its ranks scheduling-dependent).  For the scientific
 * family (profileType 2) every leaf holds a decodable payload, so every leaf is active. */
uint32_t vo_build_page_table(const vo_file* f, uint32_t* compact)
{
    uint32_t rank = 0;
    for (uint32_t leaf = 0; leaf < f->leaf_count; ++leaf) {
        const int active = f->profile_type == 2u ? 1 : ((f->payload[f->offsets[leaf]] & 3u) != 0u);
        compact[leaf] = active ? rank++ : 0xFFFFFFFFu;
    }
    return rank;
}

/* Current-frame voxel cache: 512 floats per active leaf at compact[leaf]*512, slot
 * (lz*8+ly)*8+lx; slots outside a boundary leaf's extent hold 0. */
int vo_decode_cache(const vo_file* f, int frame, const uint32_t* compact, float* cache, int threads)
{
    const uint8_t* base = (const uint8_t*)f->payload;
    int status = VO_OK;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int64_t li = 0; li < (int64_t)f->leaf_count; ++li) {
        const uint32_t leaf = (uint32_t)li;
        if (compact[leaf] == 0xFFFFFFFFu) continue;
        int bx, by, bz, w, h, d;
        leaf_geom(f, leaf, &bx, &by, &bz, &w, &h, &d);
        float vals[512];
        const uint32_t wb = f->offsets[leaf], we = f->offsets[leaf + 1];
        int st;
        float* dst = cache + (uint64_t)compact[leaf] * 512u;
        if (f->profile_type == 2u) {
            for (int i = 0; i < 512; ++i) dst[i] = 0.0f;
            for (int lz = 0; lz < d; ++lz)
                for (int ly = 0; ly < h; ++ly)
                    for (int lx = 0; lx < w; ++lx)
                        dst[(lz * 8 + ly) * 8 + lx] =
                            vo_sci_value(f, (uint32_t)(bx * 8 + lx), (uint32_t)(by * 8 + ly), (uint32_t)(bz * 8 + lz), (uint32_t)frame);
            continue;
        }
        st = vo_decode_leaf_frame(base + 4ull * wb, 4ull * (we - wb), (int)f->frames, frame, w, h, d, vals);
        if (st) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
            status = st;
            continue;
        }
        for (int i = 0; i < 512; ++i) dst[i] = 0.0f;
        for (int lz = 0; lz < d; ++lz)
            for (int ly = 0; ly < h; ++ly)
                for (int lx = 0; lx < w; ++lx) dst[(lz * 8 + ly) * 8 + lx] = vals[(lz * h + ly) * w + lx];
    }
    return status;
}

/* Point query (x,y,z,t): the value decodeFrameToDense(file, t) holds at voxel (x,y,z); the leaf
 * is found as render/src/vbt_file.cpp:250-262 leafIndexForVoxel does. */
int vo_query_points(const vo_file* f, const uint32_t* q, uint64_t n, float* out, int threads)
{
    const uint8_t* base = (const uint8_t*)f->payload;
    int status = VO_OK;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const uint32_t x = q[4 * i], y = q[4 * i + 1], z = q[4 * i + 2], t = q[4 * i + 3];
        if (f->profile_type == 2u) {
            out[i] = vo_sci_value(f, x, y, z, t);
            continue;
        }
        const uint32_t lcx = (f->width + 7u) / 8u, lcy = (f->height + 7u) / 8u, lcz = (f->depth + 7u) / 8u;
        const uint32_t bx = x / 8u < lcx - 1u ? x / 8u : lcx - 1u;
        const uint32_t by = y / 8u < lcy - 1u ? y / 8u : lcy - 1u;
        const uint32_t bz = z / 8u < lcz - 1u ? z / 8u : lcz - 1u;
        const uint32_t leaf = (bz * lcy + by) * lcx + bx;
        int gx, gy, gz, w, h, d;
        leaf_geom(f, leaf, &gx, &gy, &gz, &w, &h, &d);
        float vals[512];
        const uint32_t wb = f->offsets[leaf], we = f->offsets[leaf + 1];
        const int st = vo_decode_leaf_frame(base + 4ull * wb, 4ull * (we - wb), (int)f->frames, (int)t, w, h, d, vals);
        if (st) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
            status = st;
            out[i] = 0.0f;
            continue;
        }
        const int lx = (int)(x - bx * 8u), ly = (int)(y - by * 8u), lz = (int)(z - bz * 8u);
        out[i] = (lx < w && ly < h && lz < d) ? vals[(lz * h + ly) * w + lx] : 0.0f;
    }
    return status;
}

/* ---------------- Scientific family: render/src/scientific_decode.cpp ---------------- */

static uint32_t sci_byte(const vo_file* f, uint32_t off)
{
    const uint64_t wi = off >> 2;
    if (wi >= f->payload_words) return 0u; /* the reference throws std::out_of_range here */
    return (f->payload[wi] >> ((off & 3u) * 8u)) & 0xFFu;
}
static uint32_t sci_u16(const vo_file* f, uint32_t off) { return sci_byte(f, off) | (sci_byte(f, off + 1u) << 8); }

/* render/src/scientific_decode.cpp:61-70 decodeBfp */
static float decode_bfp(uint32_t q, float scale, int bits)
{
    if (bits <= 2) {
        static const float lv[4] = {-1.0f, -0.3333333f, 0.3333333f, 1.0f};
        return lv[q < 3u ? q : 3u] * scale;
    }
    const int levels = (1 << bits) - 1;
    const float a = (float)q / (float)levels;
    const float b = a * 2.0f;
    const float norm = b - 1.0f;
    return norm * scale;
}

/* render/src/scientific_decode.cpp:72-80 dctBasis (double evaluation, rounded to float) */
double vo_dct_basis_f64(int total, int index, int k)
{
    const double kPi = 3.14159265358979323846;
    const double invN = 1.0 / (double)total;
    const double alpha = (k == 0) ? sqrt(invN) : sqrt(2.0 * invN);
    const double arg = ((kPi / (double)total) * ((double)index + 0.5)) * (double)k;
    return alpha * cos(arg);
}
float vo_dct_basis(int total, int index, int k) { return (float)vo_dct_basis_f64(total, index, k); }

/* render/src/scientific_decode.cpp:82-97 decodeCoarseControlAt (double accumulation) */
static float sci_coarse_control(const vo_file* f, uint32_t base, int keep, int ci, int t)
{
    const uint32_t cb = base + (uint32_t)(4 + ci * (keep + 1));
    double sum = (double)vo_half_to_float((uint16_t)sci_u16(f, cb)) * (double)vo_dct_basis((int)f->frames, t, 0);
    for (int k = 1; k < keep; ++k) {
        const float scale = (uint32_t)(k - 1) < f->scale_count ? f->scales[k - 1] : 0.0f; /* reference: .at() throws */
        const float coeff = (float)(int8_t)sci_byte(f, cb + 2u + (uint32_t)(k - 1)) * scale;
        sum += (double)coeff * (double)vo_dct_basis((int)f->frames, t, k);
    }
    return (float)sum;
}

/* render/src/scientific_decode.cpp:99-123 sampleCoarseAt */
static float sci_sample_coarse(const float* ctrl, uint32_t x, uint32_t y, uint32_t z)
{
    const float fx = ((float)x / 7.0f) * 3.0f, fy = ((float)y / 7.0f) * 3.0f, fz = ((float)z / 7.0f) * 3.0f;
    int x0 = (int)floorf(fx), y0 = (int)floorf(fy), z0 = (int)floorf(fz);
    x0 = x0 < 0 ? 0 : (x0 > 2 ? 2 : x0);
    y0 = y0 < 0 ? 0 : (y0 > 2 ? 2 : y0);
    z0 = z0 < 0 ? 0 : (z0 > 2 ? 2 : z0);
    const int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
    const float tx = fx - (float)x0, ty = fy - (float)y0, tz = fz - (float)z0;
#define C(cx, cy, cz) ctrl[((cz) * 4 + (cy)) * 4 + (cx)]
    const float c00 = lerp_w(C(x0, y0, z0), C(x1, y0, z0), tx);
    const float c01 = lerp_w(C(x0, y0, z1), C(x1, y0, z1), tx);
    const float c10 = lerp_w(C(x0, y1, z0), C(x1, y1, z0), tx);
    const float c11 = lerp_w(C(x0, y1, z1), C(x1, y1, z1), tx);
#undef C
    return lerp_w(lerp_w(c00, c10, ty), lerp_w(c01, c11, ty), tz);
}

static void dense_coords(int res, uint32_t x, uint32_t y, uint32_t z, int* i0, float* tt)
{
    const uint32_t p[3] = {x, y, z};
    for (int a = 0; a < 3; ++a) {
        const float fv = ((float)p[a] / 7.0f) * (float)(res - 1);
        int v0 = (int)floorf(fv);
        v0 = v0 < 0 ? 0 : v0;
        v0 = v0 > res - 2 ? res - 2 : v0;
        i0[a] = v0;
        tt[a] = fv - (float)v0;
    }
}

static float dense_sample(const vo_file* f, uint32_t data, int res, int bits, float scale, int cx, int cy, int cz)
{
    const int ci = (cz * res + cy) * res + cx;
    const int bo = ci * bits;
    const uint32_t bi = data + (uint32_t)(bo / 8);
    const int sh = bo % 8;
    uint32_t packed = sci_byte(f, bi);
    if (sh + bits > 8) packed |= sci_byte(f, bi + 1u) << 8;
    return decode_bfp((packed >> sh) & ((1u << bits) - 1u), scale, bits);
}

static float dense_trilinear(const vo_file* f, uint32_t data, int res, int bits, float scale, const int* i0,
                             const float* tt)
{
    const int x0 = i0[0], y0 = i0[1], z0 = i0[2], x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
    const float tx = tt[0], ty = tt[1], tz = tt[2];
#define S(a, b, c) dense_sample(f, data, res, bits, scale, a, b, c)
    const float c00 = lerp_w(S(x0, y0, z0), S(x1, y0, z0), tx);
    const float c01 = lerp_w(S(x0, y0, z1), S(x1, y0, z1), tx);
    const float c10 = lerp_w(S(x0, y1, z0), S(x1, y1, z0), tx);
    const float c11 = lerp_w(S(x0, y1, z1), S(x1, y1, z1), tx);
#undef S
    return lerp_w(lerp_w(c00, c10, ty), lerp_w(c01, c11, ty), tz);
}

/* render/src/scientific_decode.cpp:125-175 decodeDenseValueAt */
static float sci_dense(const vo_file* f, uint32_t base, int keep, int res, int bits, uint32_t x, uint32_t y,
                       uint32_t z, uint32_t t)
{
    const int per = res * res * res;
    const int fbytes = (per * bits + 7) / 8;
    const uint32_t scales = base + (uint32_t)(4 + 64 * (keep + 1));
    const uint32_t data = scales + f->frames * 2u;
    const float scale = vo_half_to_float((uint16_t)sci_u16(f, scales + t * 2u));
    int i0[3];
    float tt[3];
    dense_coords(res, x, y, z, i0, tt);
    return dense_trilinear(f, data + t * (uint32_t)fbytes, res, bits, scale, i0, tt);
}

/* render/src/scientific_decode.cpp:177-233 decodeDenseTemporalBasisAt */
static float sci_dense_basis(const vo_file* f, uint32_t base, int keep, int res, int bits, int tkeep, uint32_t x,
                             uint32_t y, uint32_t z, uint32_t t)
{
    if (tkeep <= 0 || bits <= 0) return 0.0f;
    const int per = res * res * res;
    const int bbytes = (per * bits + 7) / 8;
    const uint32_t scales = base + (uint32_t)(4 + 64 * (keep + 1));
    const uint32_t data = scales + (uint32_t)(tkeep * 2);
    int i0[3];
    float tt[3];
    dense_coords(res, x, y, z, i0, tt);
    float residual = 0.0f;
    for (int k = 0; k < tkeep; ++k) {
        const float scale = vo_half_to_float((uint16_t)sci_u16(f, scales + (uint32_t)(k * 2)));
        const float tri = dense_trilinear(f, data + (uint32_t)(k * bbytes), res, bits, scale, i0, tt);
        const float term = tri * vo_dct_basis((int)f->frames, (int)t, k);
        residual = residual + term;
    }
    return residual;
}

/* render/src/scientific_decode.cpp:235-295 decodeSparseResidualAt */
static float sci_sparse(const vo_file* f, uint32_t base, uint32_t hdr, int keep, uint32_t li, uint32_t t)
{
    const uint32_t count = (hdr >> 16) & 0x0FFFu;
    if (count == 0u) return 0.0f;
    const uint32_t tier = (hdr >> 8) & 3u;
    const uint32_t cap = tier == 0u ? 64u : tier == 1u ? 256u : tier == 2u ? 768u : 1024u;
    const uint32_t fpb = ((hdr >> 10) & 0xFu) + 1u;
    const uint32_t bin = t / fpb < 15u ? t / fpb : 15u;
    const uint32_t lt = (t - bin * fpb) & 0xFFu;
    const uint32_t sb = base + 4u + (uint32_t)(64 * (keep + 1));
    const uint32_t sw = sci_byte(f, sb) | (sci_byte(f, sb + 1) << 8) | (sci_byte(f, sb + 2) << 16) | (sci_byte(f, sb + 3) << 24);
    float es;
    memcpy(&es, &sw, 4);
    if (!(es > 0.0f)) return 0.0f;
    const uint32_t mo = sb + 4u + ((li >> 5) * 4u);
    const uint32_t mw = sci_byte(f, mo) | (sci_byte(f, mo + 1) << 8) | (sci_byte(f, mo + 2) << 16) | (sci_byte(f, mo + 3) << 24);
    if ((mw & (1u << (li & 31u))) == 0u) return 0.0f;
    const uint32_t bb = sb + 4u + 64u;
    const uint32_t start = sci_u16(f, bb + bin * 2u);
    const uint32_t end = bin + 1u < 16u ? sci_u16(f, bb + (bin + 1u) * 2u) : (count & 0xFFFFu);
    if (start >= end) return 0.0f;
    const uint32_t cb = bb + 32u, rb = cb + cap * 2u;
    const uint32_t target = ((lt << 9) | (li & 0x1FFu)) & 0xFFFFu;
    int left = (int)start, right = (int)end - 1;
    while (left <= right) {
        const int mid = (left + right) >> 1;
        const uint32_t key = sci_u16(f, cb + (uint32_t)mid * 2u);
        if (key == target) {
            const uint32_t byte = sci_byte(f, rb + (uint32_t)(mid >> 1));
            const uint32_t nib = (mid & 1) == 0 ? (byte & 0xFu) : ((byte >> 4) & 0xFu);
            int q = (int)nib;
            if (q & 8) q -= 16;
            return (float)q * es;
        }
        if (key < target) left = mid + 1;
        else right = mid - 1;
    }
    return 0.0f;
}

/* render/src/scientific_decode.cpp:297-331 decodeScientificResidualAt */
static float sci_residual(const vo_file* f, uint32_t base, uint32_t hdr, int keep, uint32_t li, uint32_t lx,
                          uint32_t ly, uint32_t lz, uint32_t t)
{
    const uint32_t mode = hdr & 3u;
    if (mode == 0u) return 0.0f;
    if (mode == 1u) return sci_sparse(f, base, hdr, keep, li, t);
    const int res = mode == 2u ? 3 : 4;
    const int bits = (int)((hdr >> 8) & 0xFu);
    const uint32_t sub = (hdr >> 12) & 7u;
    const int tkeep = (int)((hdr >> 15) & 0xFu) + 1;
    return sub == 1u ? sci_dense_basis(f, base, keep, res, bits, tkeep, lx, ly, lz, t)
                     : sci_dense(f, base, keep, res, bits, lx, ly, lz, t);
}

static uint32_t sci_leaf_for(const vo_file* f, uint32_t x, uint32_t y, uint32_t z)
{
    const uint32_t lcx = (f->width + 7u) / 8u, lcy = (f->height + 7u) / 8u, lcz = (f->depth + 7u) / 8u;
    const uint32_t bx = x / 8u < lcx - 1u ? x / 8u : lcx - 1u;
    const uint32_t by = y / 8u < lcy - 1u ? y / 8u : lcy - 1u;
    const uint32_t bz = z / 8u < lcz - 1u ? z / 8u : lcz - 1u;
    return (bz * lcy + by) * lcx + bx;
}

/* render/src/scientific_decode.cpp:335-359 decodeScientificValueAtCpu */
float vo_sci_value(const vo_file* f, uint32_t x, uint32_t y, uint32_t z, uint32_t t)
{
    const uint32_t leaf = sci_leaf_for(f, x, y, z);
    const uint32_t wo = f->offsets[leaf];
    const uint32_t hdr = wo < f->payload_words ? f->payload[wo] : 0u;
    const uint32_t base = wo * 4u;
    const uint32_t lx = x % 8u, ly = y % 8u, lz = z % 8u;
    const uint32_t li = (lz * 8u + ly) * 8u + lx;
    const int keep = (int)((hdr >> 2) & 0x3Fu) + 1;
    float ctrl[64];
    for (int i = 0; i < 64; ++i) ctrl[i] = sci_coarse_control(f, base, keep, i, (int)t);
    const float coarse = sci_sample_coarse(ctrl, lx, ly, lz);
    return coarse + sci_residual(f, base, hdr, keep, li, lx, ly, lz, t);
}

/* render/src/scientific_decode.cpp:361-409 reconstructScientificFrameCpu */
void vo_sci_frame(const vo_file* f, uint32_t frame, float* out, int threads)
{
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int64_t li = 0; li < (int64_t)f->leaf_count; ++li) {
        const uint32_t leaf = (uint32_t)li;
        int bx, by, bz, w, h, d;
        leaf_geom(f, leaf, &bx, &by, &bz, &w, &h, &d);
        const uint32_t wo = f->offsets[leaf];
        const uint32_t hdr = wo < f->payload_words ? f->payload[wo] : 0u;
        const uint32_t base = wo * 4u;
        const int keep = (int)((hdr >> 2) & 0x3Fu) + 1;
        float ctrl[64];
        for (int i = 0; i < 64; ++i) ctrl[i] = sci_coarse_control(f, base, keep, i, (int)frame);
        for (int lz = 0; lz < d; ++lz)
            for (int ly = 0; ly < h; ++ly)
                for (int lx = 0; lx < w; ++lx) {
                    const uint32_t lidx = (uint32_t)((lz * 8 + ly) * 8 + lx);
                    const float c = sci_sample_coarse(ctrl, (uint32_t)lx, (uint32_t)ly, (uint32_t)lz);
                    const float r = sci_residual(f, base, hdr, keep, lidx, (uint32_t)lx, (uint32_t)ly, (uint32_t)lz, frame);
                    out[((uint64_t)(bz * 8 + lz) * f->height + (uint64_t)(by * 8 + ly)) * f->width + (uint64_t)(bx * 8 + lx)] = c + r;
                }
    }
}

void vo_sci_query_points(const vo_file* f, const uint32_t* q, uint64_t n, float* out, int threads)
{
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) out[i] = vo_sci_value(f, q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]);
}
