// capi.cu -- the C-ABI (include/vbt_b200.h): asset registry, reader validation, uploads, launches.
//
// Assets stay resident in device memory: offsets + payload words as read from the file, the AC
// scale table, a host-built DCT basis table for scientific assets, and the walker's leaf table +
// page table.  Every decode call is asynchronous on the caller's stream; decode errors are
// recorded on the device (lowest failing leaf wins) and read by vbt_asset_sync_status.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/vbt_b200.h"
#include "asset.h"
#include "kernels.cuh"

namespace vbtb {
void launch_checked_decode(const uint8_t* stream, uint32_t bytes, uint32_t codec, uint32_t cc, uint32_t bins,
                           uint32_t kf, int align, int total, const uint32_t* ci, const int32_t* fr, uint64_t n,
                           float* out, int32_t* status, cudaStream_t st);
}

using namespace vbtb;


namespace {

thread_local std::string g_err;

int fail(int status, const std::string& msg)
{
    g_err = msg;
    return status;
}

int cuda_fail(cudaError_t e, const char* what)
{
    return fail(VBT_STATUS_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CUDA_TRY(expr)                                     \
    do {                                                   \
        const cudaError_t e_ = (expr);                     \
        if (e_ != cudaSuccess) return cuda_fail(e_, #expr); \
    } while (0)

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

uint32_t rd32(const uint8_t* p)
{
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}

// Reader rules and messages of render/src/vbt_file.cpp:39-206, on an in-memory file image.
int validate_image(const uint8_t* b, uint64_t len, vbt_header* h)
{
    const uint64_t kHeader = 52;
    if (len < kHeader) return fail(VBT_STATUS_FILE, "Invalid VBTPACK4 file size.");
    uint32_t f[11];
    for (int i = 0; i < 11; ++i) f[i] = rd32(b + 8 + 4 * i);
    *h = vbt_header{f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], f[10]};
    if (std::memcmp(b, "VBTPACK4", 8) != 0) return fail(VBT_STATUS_FILE, "Unsupported magic. Expected VBTPACK4.");
    if (h->version != 4u) return fail(VBT_STATUS_FILE, "Unsupported VBTPACK4 version: " + std::to_string(h->version));
    if (!h->width || !h->height || !h->depth || !h->frames)
        return fail(VBT_STATUS_FILE, "VBTPACK4 dimensions and frame count must be non-zero.");
    if (h->leaf_size != 8u) return fail(VBT_STATUS_FILE, "VBTPACK4 v4 requires leafSize=8.");
    if (h->coarse_resolution == 0u || h->coarse_resolution > 8u)
        return fail(VBT_STATUS_FILE, "Invalid VBTPACK4 coarse resolution.");
    if (h->profile_type > 2u) return fail(VBT_STATUS_FILE, "Invalid VBTPACK4 profile type.");
    if (h->max_coarse_keep > h->frames || h->coarse_ac_scale_count > 64u ||
        h->coarse_ac_scale_count > h->max_coarse_keep)
        return fail(VBT_STATUS_FILE, "Invalid VBTPACK4 coarse temporal metadata.");
    const uint64_t lx = ((uint64_t)h->width + 7) / 8, ly = ((uint64_t)h->height + 7) / 8, lz = ((uint64_t)h->depth + 7) / 8;
    const uint64_t expect = lx * ly * lz;
    if (expect > 0xFFFFFFFFull) return fail(VBT_STATUS_FILE, "VBTPACK4 leaf count overflows the v4 header.");
    if (h->leaf_count != expect) return fail(VBT_STATUS_FILE, "VBTPACK4 leafCount does not match dimensions and leafSize.");
    const uint64_t tables = kHeader + 4ull * h->coarse_ac_scale_count + 4ull * ((uint64_t)h->leaf_count + 1u);
    if (tables > len) return fail(VBT_STATUS_FILE, "VBTPACK4 file is truncated before its offset table.");
    const uint8_t* off = b + kHeader + 4ull * h->coarse_ac_scale_count;
    if (rd32(off) != 0u) return fail(VBT_STATUS_FILE, "VBTPACK4 offset table must begin at word zero.");
    for (uint64_t i = 0; i < h->leaf_count; ++i)
        if (rd32(off + 4 * i) >= rd32(off + 4 * (i + 1)))
            return fail(VBT_STATUS_FILE, "VBTPACK4 offsets must be strictly increasing for every leaf.");
    const uint64_t words = rd32(off + 4ull * h->leaf_count);
    const uint64_t total = tables + 4ull * words;
    if (total != len)
        return fail(VBT_STATUS_FILE, total > len ? "VBTPACK4 payload is truncated." : "VBTPACK4 file contains trailing bytes.");
    return VBT_STATUS_OK;
}

std::once_flag g_tables_once[64];

int ensure_device(int device)
{
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(VBT_STATUS_CUDA, "no usable CUDA device for the VBT decode path");
    if (device < 0 || device >= n || device >= 64) return fail(VBT_STATUS_INVALID_ARGUMENT, "device index out of range");
    return VBT_STATUS_OK;
}

int alloc(vbt_asset* a, void** p, size_t bytes)
{
    const cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
    a->allocations.push_back(*p);
    a->device_bytes += bytes;
    return VBT_STATUS_OK;
}

void free_all(vbt_asset* a)
{
    for (void* p : a->allocations) cudaFree(p);
    a->allocations.clear();
    if (a->stage_in) cudaFree(a->stage_in);
    if (a->stage_out) cudaFree(a->stage_out);
}

int grow(void** p, size_t* have, size_t need)
{
    if (*have >= need) return VBT_STATUS_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *have = 0;
    const cudaError_t e = cudaMalloc(p, need);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc staging");
    *have = need;
    return VBT_STATUS_OK;
}

int check_launch(const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, what);
    return VBT_STATUS_OK;
}

}  // namespace

namespace vbtb {
// Message for vbt_last_error() from other translation units of the library.
int set_last_error(int status, const std::string& msg) { return fail(status, msg); }
}  // namespace vbtb

// Launch-shape facts taken from a render-temporal image's route tags and leaf sizes (nothing is
// read from the device):
//  - sparse: fewer than half of the leaves non-EMPTY (the point-query kernel's shape hint);
//  - the shared-memory leaf stage of the render decode kernel: the largest 16-byte-aligned window
//    of a non-EMPTY leaf, capped so that two CTAs fit on an SM (232,448 B of shared memory per SM
//    less 1 KiB per CTA); an asset with bigger leaves gets the kernel variant that decodes those
//    from global memory.  When more than a quarter of the non-EMPTY leaves exceed the cap, no leaf
//    is staged: the kernel then reads every leaf through L1, which the unused stage leaves free.
// Computed at creation and again for every re-uploaded image, whose leaves may differ in size.
static void image_shape(const vbt_header& h, const uint8_t* b, uint64_t off_off, uint64_t pay_off, uint64_t words,
                        AssetGeom& g, bool& sparse)
{
    if (h.profile_type == 2u) return;
    const uint8_t* off = b + off_off;
    const uint32_t cap = ((233472u / 2u - 1024u - kLeafFixedBytes - 16u) / 1024u) * 1024u;
    uint64_t active = 0, maxw = 0, fits = 0;
    for (uint32_t i = 0; i < h.leaf_count; ++i) {
        const uint64_t w0 = rd32(off + 4ull * i), w1 = rd32(off + 4ull * (i + 1));
        if (w1 <= w0 || w0 >= words || (rd32(b + pay_off + 4ull * w0) & 3u) == 0u) continue;
        ++active;
        const uint64_t a0 = (4ull * w0) & ~15ull, a1 = (4ull * w1 + 15u) & ~15ull;
        maxw = std::max(maxw, a1 - a0);
        fits += a1 - a0 <= cap ? 1u : 0u;
    }
    sparse = 2u * active < (uint64_t)h.leaf_count;
    g.sparse = sparse ? 1u : 0u;
    g.max_window = (uint32_t)std::min<uint64_t>(maxw, 0xFFFFFFFFull);
    g.stage_bytes = std::min<uint32_t>(std::max<uint32_t>((g.max_window + 1023u) & ~1023u, 4096u), cap);
    if (4u * fits < 3u * active) g.stage_bytes = 0u;
}

extern "C" {

const char* vbt_status_string(int s)
{
    switch (s) {
    case VBT_STATUS_OK: return "ok";
    case VBT_STATUS_LEAF_TOO_SMALL: return "render temporal leaf bytes too small";
    case VBT_STATUS_PREFIX_MISSING: return "render temporal leaf prefix missing";
    case VBT_STATUS_LEAF_SHORT: return "render temporal leaf shorter than computed layout";
    case VBT_STATUS_SHELL_OCC_OOB: return "render temporal shell occupancy is out of bounds";
    case VBT_STATUS_SHELL_GROUP_PREFIX: return "render temporal shell group prefix is inconsistent";
    case VBT_STATUS_SHELL_NO_ACTIVE: return "render temporal shell mode contains no active voxels";
    case VBT_STATUS_SHELL_RESIDUAL_OOB: return "render temporal shell residual stream is out of bounds";
    case VBT_STATUS_SHELL_TRAILING: return "render temporal shell leaf contains trailing bytes";
    case VBT_STATUS_CONTROL_INDEX: return "render temporal control index out of range";
    case VBT_STATUS_STREAM_OOB: return "render temporal stream decode out of bounds";
    case VBT_STATUS_DECODE_OOB: return "render temporal decode out of bounds";
    case VBT_STATUS_KEY_RANGE_OOB: return "render temporal keyframe range out of bounds";
    case VBT_STATUS_KEY_INDEX: return "render temporal keyframe index out of range";
    case VBT_STATUS_WAIT_TIMEOUT: return "device-side wait timed out";
    case VBT_STATUS_INVALID_ARGUMENT: return "invalid argument";
    case VBT_STATUS_FILE: return "invalid VBTPACK4 file";
    case VBT_STATUS_CUDA: return "CUDA error";
    case VBT_STATUS_LIMIT: return "request exceeds a fixed capacity";
    case VBT_STATUS_UNSUPPORTED: return "leaf mode not covered by this call";
    default: return "unknown status";
    }
}

const char* vbt_last_error(void) { return g_err.c_str(); }

int vbt_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

int vbt_validate_file_image(const void* bytes, uint64_t len, vbt_header* out)
{
    if (!bytes || !out) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    return validate_image(static_cast<const uint8_t*>(bytes), len, out);
}

int vbt_asset_create(const void* file_bytes, uint64_t len, int device, vbt_asset** out)
{
    if (!file_bytes || !out) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    vbt_header h{};
    int st = validate_image(static_cast<const uint8_t*>(file_bytes), len, &h);
    if (st) return st;
    if ((st = ensure_device(device))) return st;
    DeviceGuard guard(device);
    std::call_once(g_tables_once[device], [] { upload_axis_tables(); });
    CUDA_TRY(cudaGetLastError());

    auto* a = new vbt_asset();
    a->device = device;
    a->hdr = h;
    const uint8_t* b = static_cast<const uint8_t*>(file_bytes);
    const uint64_t scale_off = 52, off_off = scale_off + 4ull * h.coarse_ac_scale_count;
    const uint64_t pay_off = off_off + 4ull * ((uint64_t)h.leaf_count + 1u);
    const uint64_t words = (len - pay_off) / 4u;
    AssetGeom& g = a->dev.g;
    g.width = h.width;
    g.height = h.height;
    g.depth = h.depth;
    g.frames = h.frames;
    g.lcx = (h.width + 7) / 8;
    g.lcy = (h.height + 7) / 8;
    g.lcz = (h.depth + 7) / 8;
    g.leaf_count = h.leaf_count;
    g.profile = h.profile_type;
    g.scale_count = h.coarse_ac_scale_count;
    g.payload_words = words;
    image_shape(h, b, off_off, pay_off, words, g, a->sparse);
    const uint32_t L = h.leaf_count;
    const uint32_t tiles = (L + kWalkTile - 1) / kWalkTile;
    void *d_off, *d_pay, *d_scales, *d_basis, *d_entries, *d_compact, *d_list, *d_counters, *d_err, *d_tiles, *d_sorted,
        *d_work;
    // payload gets 16 bytes of tail padding so vector reads near the end stay inside the allocation
    if ((st = alloc(a, &d_off, 4ull * (L + 1))) || (st = alloc(a, &d_pay, 4ull * words + 16)) ||
        (st = alloc(a, &d_scales, 4ull * (h.coarse_ac_scale_count + 1))) ||
        (st = alloc(a, &d_basis, h.profile_type == 2u ? 4ull * h.frames * 64u : 16u)) ||
        (st = alloc(a, &d_entries, sizeof(LeafEntry) * (uint64_t)L)) || (st = alloc(a, &d_compact, 4ull * L)) ||
        (st = alloc(a, &d_list, 4ull * L)) || (st = alloc(a, &d_counters, 16)) || (st = alloc(a, &d_err, 8)) ||
        (st = alloc(a, &d_tiles, 8ull * tiles)) || (st = alloc(a, &d_sorted, L)) ||
        (st = alloc(a, &d_work, 8ull * kWorkSlots)) || (st = alloc(a, reinterpret_cast<void**>(&a->d_stats), 32))) {
        free_all(a);
        delete a;
        return st;
    }
    cudaMemcpy(d_off, b + off_off, 4ull * (L + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(d_pay, b + pay_off, 4ull * words, cudaMemcpyHostToDevice);
    cudaMemset(static_cast<uint8_t*>(d_pay) + 4ull * words, 0, 16);
    cudaMemset(d_scales, 0, 4ull * (h.coarse_ac_scale_count + 1));
    if (h.coarse_ac_scale_count) cudaMemcpy(d_scales, b + scale_off, 4ull * h.coarse_ac_scale_count, cudaMemcpyHostToDevice);
    if (h.profile_type == 2u) {
        // DCT-II basis b_k(t) = alpha_k cos(pi/T (t + 1/2) k), evaluated in double and rounded to
        // float exactly as render/src/scientific_decode.cpp:72-80 (dctBasis) does.
        std::vector<float> basis((size_t)h.frames * 64u);
        const double kPi = 3.14159265358979323846;
        const double invN = 1.0 / (double)h.frames;
        for (uint32_t t = 0; t < h.frames; ++t)
            for (int k = 0; k < 64; ++k) {
                const double alpha = (k == 0) ? std::sqrt(invN) : std::sqrt(2.0 * invN);
                const double arg = ((kPi / (double)h.frames) * ((double)t + 0.5)) * (double)k;
                basis[(size_t)t * 64 + k] = (float)(alpha * std::cos(arg));
            }
        cudaMemcpy(d_basis, basis.data(), basis.size() * 4, cudaMemcpyHostToDevice);
    }
    cudaMemset(d_counters, 0, 16);
    cudaMemset(d_err, 0xFF, 8);
    cudaMemset(d_tiles, 0, 8ull * tiles);
    cudaMemset(d_sorted, 0, L);
    cudaMemset(d_work, 0, 8ull * kWorkSlots);
    const cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) {
        free_all(a);
        delete a;
        return cuda_fail(ce, "asset upload");
    }
    DeviceAsset& d = a->dev;
    d.offsets = static_cast<const uint32_t*>(d_off);
    d.payload = static_cast<const uint32_t*>(d_pay);
    d.scales = static_cast<const float*>(d_scales);
    d.basis = static_cast<const float*>(d_basis);
    d.entries = static_cast<LeafEntry*>(d_entries);
    d.compact = static_cast<uint32_t*>(d_compact);
    d.active_list = static_cast<uint32_t*>(d_list);
    d.counters = static_cast<uint32_t*>(d_counters);
    d.err = static_cast<unsigned long long*>(d_err);
    d.tile_state = static_cast<unsigned long long*>(d_tiles);
    d.key_sorted = static_cast<uint8_t*>(d_sorted);
    d.work = static_cast<unsigned long long*>(d_work);
    // first page-table build and key-order analysis, synchronously, so that a returned asset is
    // ready to decode
    launch_walk(d, ++a->epoch, 0);
    launch_key_order(d, 0);
    const cudaError_t we = cudaDeviceSynchronize();
    if (we != cudaSuccess) {
        free_all(a);
        delete a;
        return cuda_fail(we, "page table build");
    }
    *out = a;
    return VBT_STATUS_OK;
}

int vbt_asset_open(const char* path, int device, vbt_asset** out)
{
    if (!path || !out) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return fail(VBT_STATUS_FILE, std::string("Failed to query file size: ") + path);
    std::fseek(fp, 0, SEEK_END);
    const long n = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    std::vector<uint8_t> bytes(n > 0 ? (size_t)n : 0);
    const size_t got = n > 0 ? std::fread(bytes.data(), 1, bytes.size(), fp) : 0;
    std::fclose(fp);
    if (got != bytes.size()) return fail(VBT_STATUS_FILE, "Failed to read VBTPACK header.");
    return vbt_asset_create(bytes.data(), bytes.size(), device, out);
}

int vbt_asset_upload(vbt_asset* a, const void* file_bytes, uint64_t len, void* stream)
{
    if (!a || !file_bytes) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    const uint8_t* b = static_cast<const uint8_t*>(file_bytes);
    if (len < 52 || std::memcmp(b, &"VBTPACK4"[0], 8) != 0) return fail(VBT_STATUS_FILE, "Unsupported magic. Expected VBTPACK4.");
    uint32_t f[11];
    for (int i = 0; i < 11; ++i) f[i] = rd32(b + 8 + 4 * i);
    const vbt_header& h = a->hdr;
    const uint32_t want[11] = {h.version, h.width, h.height, h.depth, h.frames, h.leaf_size, h.coarse_resolution,
                               h.max_coarse_keep, h.leaf_count, h.profile_type, h.coarse_ac_scale_count};
    if (std::memcmp(f, want, sizeof f) != 0) return fail(VBT_STATUS_INVALID_ARGUMENT, "image header differs from the asset's");
    const uint64_t off_off = 52 + 4ull * h.coarse_ac_scale_count;
    const uint64_t pay_off = off_off + 4ull * ((uint64_t)h.leaf_count + 1u);
    if (len != pay_off + 4ull * a->dev.g.payload_words)
        return fail(VBT_STATUS_INVALID_ARGUMENT, "image size differs from the asset's");
    // the new image's leaves may be larger than the old ones: the stage and the kernel variant
    // follow the image, and timeline graphs captured with the old shape are dropped
    AssetGeom g = a->dev.g;
    bool sparse = a->sparse;
    image_shape(h, b, off_off, pay_off, a->dev.g.payload_words, g, sparse);
    DeviceGuard guard(a->device);
    if (g.stage_bytes != a->dev.g.stage_bytes || g.max_window != a->dev.g.max_window) release_timeline_graphs(a);
    a->dev.g = g;
    a->sparse = sparse;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (h.coarse_ac_scale_count)
        CUDA_TRY(cudaMemcpyAsync((void*)a->dev.scales, b + 52, 4ull * h.coarse_ac_scale_count, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync((void*)a->dev.offsets, b + off_off, 4ull * ((uint64_t)h.leaf_count + 1u), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync((void*)a->dev.payload, b + pay_off, 4ull * a->dev.g.payload_words, cudaMemcpyHostToDevice, s));
    // the key-order analysis belongs to the payload: redo it (it needs a walked leaf table)
    launch_walk(a->dev, ++a->epoch, s);
    launch_key_order(a->dev, s);
    return check_launch("key_order_kernel");
}

int vbt_asset_destroy(vbt_asset* a)
{
    if (!a) return VBT_STATUS_OK;
    {
        DeviceGuard guard(a->device);
        release_timeline_graphs(a);
        free_all(a);
    }
    delete a;
    return VBT_STATUS_OK;
}

int vbt_asset_get_info(vbt_asset* a, vbt_asset_info* info)
{
    if (!a || !info) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    DeviceGuard guard(a->device);
    std::memset(info, 0, sizeof *info);
    info->header = a->hdr;
    info->leaf_count_x = a->dev.g.lcx;
    info->leaf_count_y = a->dev.g.lcy;
    info->leaf_count_z = a->dev.g.lcz;
    info->payload_words = a->dev.g.payload_words;
    info->device_bytes = a->device_bytes;
    info->device = a->device;
    CUDA_TRY(cudaMemcpy(&info->active_leaf_count, a->dev.counters, 4, cudaMemcpyDeviceToHost));
    return VBT_STATUS_OK;
}

int vbt_build_page_table(vbt_asset* a, void* stream)
{
    if (!a) return fail(VBT_STATUS_INVALID_ARGUMENT, "null asset");
    DeviceGuard guard(a->device);
    // the leaf table was built by the walker when the payload was uploaded; a page table needs
    // only each row's active flag
    launch_page_table(a->dev, ++a->epoch, static_cast<cudaStream_t>(stream));
    return check_launch("page_table_kernel");
}

int vbt_page_table_device(vbt_asset* a, const uint32_t** c, const uint32_t** l, const uint32_t** n)
{
    if (!a) return fail(VBT_STATUS_INVALID_ARGUMENT, "null asset");
    if (c) *c = a->dev.compact;
    if (l) *l = a->dev.active_list;
    if (n) *n = a->dev.counters;
    return VBT_STATUS_OK;
}

int vbt_get_page_table(vbt_asset* a, uint32_t* compact, uint32_t* active)
{
    if (!a) return fail(VBT_STATUS_INVALID_ARGUMENT, "null asset");
    DeviceGuard guard(a->device);
    CUDA_TRY(cudaDeviceSynchronize());
    if (compact) CUDA_TRY(cudaMemcpy(compact, a->dev.compact, 4ull * a->hdr.leaf_count, cudaMemcpyDeviceToHost));
    if (active) CUDA_TRY(cudaMemcpy(active, a->dev.counters, 4, cudaMemcpyDeviceToHost));
    return VBT_STATUS_OK;
}

int vbt_get_leaf_table(vbt_asset* a, uint32_t* rows)
{
    if (!a || !rows) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    DeviceGuard guard(a->device);
    CUDA_TRY(cudaDeviceSynchronize());
    CUDA_TRY(cudaMemcpy(rows, a->dev.entries, sizeof(LeafEntry) * (uint64_t)a->hdr.leaf_count, cudaMemcpyDeviceToHost));
    return VBT_STATUS_OK;
}

static int check_frames(vbt_asset* a, const int* frames, int nframes)
{
    if (!frames || nframes <= 0 || nframes > kMaxLaunchFrames)
        return fail(VBT_STATUS_INVALID_ARGUMENT, "need 1..128 frames");
    if (a->hdr.profile_type == 2u)
        for (int i = 0; i < nframes; ++i)
            if (frames[i] < 0 || (uint32_t)frames[i] >= a->hdr.frames)
                return fail(VBT_STATUS_INVALID_ARGUMENT, "scientific frame index outside [0, frames)");
    return VBT_STATUS_OK;
}

int vbt_decode_cache(vbt_asset* a, const int* frames, int nframes, float* out, uint64_t stride, int grid, void* stream)
{
    if (!a || !out) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    int st = check_frames(a, frames, nframes);
    if (st) return st;
    DeviceGuard guard(a->device);
    launch_decode_cache(a->dev, a->launch_seq.fetch_add(1), frames, nframes, out, stride, grid, static_cast<cudaStream_t>(stream));
    return check_launch("decode_kernel<cache>");
}

int vbt_decode_control_cache(vbt_asset* a, const int* frames, int nframes, float* out, uint64_t stride, void* stream)
{
    if (!a || !out) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (a->hdr.profile_type == 2u)
        return fail(VBT_STATUS_INVALID_ARGUMENT, "the control cache covers render-temporal assets");
    int st = check_frames(a, frames, nframes);
    if (st) return st;
    DeviceGuard guard(a->device);
    launch_control_cache(a->dev, frames, nframes, out, stride, static_cast<cudaStream_t>(stream));
    return check_launch("control_cache_kernel");
}

int vbt_decode_cache_plain(vbt_asset* a, int frame, float* out, void* stream)
{
    if (!a || !out) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    int st = check_frames(a, &frame, 1);
    if (st) return st;
    DeviceGuard guard(a->device);
    launch_decode_cache_plain(a->dev, frame, out, static_cast<cudaStream_t>(stream));
    return check_launch("decode_plain_kernel");
}

int vbt_decode_frames(vbt_asset* a, const int* frames, int nframes, float* out, int grid, void* stream)
{
    if (!a || !out) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    int st = check_frames(a, frames, nframes);
    if (st) return st;
    DeviceGuard guard(a->device);
    launch_decode_dense(a->dev, a->launch_seq.fetch_add(1), frames, nframes, out, grid, static_cast<cudaStream_t>(stream));
    return check_launch("decode_kernel<dense>");
}

int vbt_query_points(vbt_asset* a, const uint32_t* q, uint64_t n, float* out, void* stream)
{
    if (!a || (n && (!q || !out))) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (((uintptr_t)q & 15u) != 0u) return fail(VBT_STATUS_INVALID_ARGUMENT, "query buffer must be 16-byte aligned");
    DeviceGuard guard(a->device);
    launch_query_points(a->dev, q, n, out, a->sparse, static_cast<cudaStream_t>(stream));
    return check_launch("query_points_kernel");
}

int vbt_query_slice(vbt_asset* a, uint32_t z, int t0, int t1, float* out, void* stream)
{
    if (!a || !out) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (z >= a->hdr.depth || t1 < t0) return fail(VBT_STATUS_INVALID_ARGUMENT, "slice outside the volume");
    if (a->hdr.profile_type == 2u && (t0 < 0 || (uint32_t)t1 > a->hdr.frames))
        return fail(VBT_STATUS_INVALID_ARGUMENT, "scientific frame range outside [0, frames)");
    DeviceGuard guard(a->device);
    launch_query_slice(a->dev, z, t0, t1, out, static_cast<cudaStream_t>(stream));
    return check_launch("query_slice_kernel");
}

int vbt_asset_sync_status(vbt_asset* a, void* stream, uint32_t* bad_leaf)
{
    if (!a) return fail(VBT_STATUS_INVALID_ARGUMENT, "null asset");
    DeviceGuard guard(a->device);
    CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    unsigned long long v = ~0ull;
    CUDA_TRY(cudaMemcpy(&v, a->dev.err, 8, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemset(a->dev.err, 0xFF, 8));
    if (v == ~0ull) {
        if (bad_leaf) *bad_leaf = 0xFFFFFFFFu;
        return VBT_STATUS_OK;
    }
    const uint32_t leaf = (uint32_t)(v >> 8), code = (uint32_t)(v & 0xFFu);
    if (bad_leaf) *bad_leaf = leaf;
    return fail((int)code, std::string(vbt_status_string((int)code)) + " (leaf " + std::to_string(leaf) + ")");
}

int vbt_query_points_host(vbt_asset* a, const uint32_t* q, uint64_t n, float* out, void* stream)
{
    if (!a || (n && (!q || !out))) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (n == 0) return VBT_STATUS_OK;
    DeviceGuard guard(a->device);
    std::lock_guard<std::mutex> lock(a->mu);
    int st;
    if ((st = grow(&a->stage_in, &a->stage_in_bytes, 16ull * n)) || (st = grow(&a->stage_out, &a->stage_out_bytes, 4ull * n)))
        return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CUDA_TRY(cudaMemcpyAsync(a->stage_in, q, 16ull * n, cudaMemcpyHostToDevice, s));
    launch_query_points(a->dev, static_cast<const uint32_t*>(a->stage_in), n, static_cast<float*>(a->stage_out),
                        a->sparse, s);
    if ((st = check_launch("query_points_kernel"))) return st;
    CUDA_TRY(cudaMemcpyAsync(out, a->stage_out, 4ull * n, cudaMemcpyDeviceToHost, s));
    return vbt_asset_sync_status(a, stream, nullptr);
}

int vbt_decode_frames_host(vbt_asset* a, const int* frames, int nframes, float* out, void* stream)
{
    if (!a || !out) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    int st = check_frames(a, frames, nframes);
    if (st) return st;
    DeviceGuard guard(a->device);
    std::lock_guard<std::mutex> lock(a->mu);
    const uint64_t vox = (uint64_t)a->hdr.width * a->hdr.height * a->hdr.depth;
    if ((st = grow(&a->stage_out, &a->stage_out_bytes, 4ull * vox * nframes))) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    launch_decode_dense(a->dev, a->launch_seq.fetch_add(1), frames, nframes, static_cast<float*>(a->stage_out), 0, s);
    if ((st = check_launch("decode_kernel<dense>"))) return st;
    CUDA_TRY(cudaMemcpyAsync(out, a->stage_out, 4ull * vox * nframes, cudaMemcpyDeviceToHost, s));
    return vbt_asset_sync_status(a, stream, nullptr);
}

int vbt_decode_window(vbt_asset* a, int t0, int n, float* d_out, uint64_t frame_stride, void* stream)
{
    if (!a || !d_out) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (a->hdr.profile_type == 2u) {
        if (n < 1 || n > 64 || t0 < 0 || (uint64_t)t0 + (uint64_t)n > a->hdr.frames)
            return fail(VBT_STATUS_INVALID_ARGUMENT, "window must be 1..64 frames inside [0, frames)");
        if (frame_stride < 512ull * a->hdr.leaf_count)
            return fail(VBT_STATUS_INVALID_ARGUMENT, "frame_stride below leaf_count * 512");
        DeviceGuard guard(a->device);
        launch_sci_window(a->dev, t0, n, d_out, frame_stride, static_cast<cudaStream_t>(stream));
        return check_launch("sci_window_kernel");
    }
    if (n < 1 || n > 64 || t0 < 0 || (uint64_t)t0 + (uint64_t)n > a->hdr.frames)
        return fail(VBT_STATUS_INVALID_ARGUMENT, "render windows must cover 1..64 frames inside [0, frames)");
    if ((reinterpret_cast<uintptr_t>(d_out) & 15u) != 0u || (frame_stride & 3u) != 0u)
        return fail(VBT_STATUS_INVALID_ARGUMENT, "output must be 16-byte aligned, frame_stride a multiple of 4");
    DeviceGuard guard(a->device);
    launch_render_window(a->dev, a->launch_seq.fetch_add(1), t0, n, d_out, frame_stride,
                         static_cast<cudaStream_t>(stream));
    return check_launch("render_window_kernel");
}

int vbt_window_error(vbt_asset* a, int t0, int n, const float* d_values, uint64_t frame_stride, double* stats,
                     void* stream)
{
    if (!a || !d_values || !stats) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (n < 1 || t0 < 0 || (uint64_t)t0 + (uint64_t)n > a->hdr.frames)
        return fail(VBT_STATUS_INVALID_ARGUMENT, "frames outside [0, frames)");
    DeviceGuard guard(a->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool sci = a->hdr.profile_type == 2u;
    if (sci) launch_sci_window_oracle(a->dev, t0, n, d_values, frame_stride, a->d_stats, s);
    else launch_render_window_oracle(a->dev, t0, n, d_values, frame_stride, a->d_stats, s);
    int st;
    if ((st = check_launch(sci ? "sci_window_oracle_kernel" : "render_window_oracle_kernel"))) return st;
    unsigned long long raw[4];
    uint32_t leaves = a->hdr.leaf_count;
    CUDA_TRY(cudaMemcpyAsync(raw, a->d_stats, sizeof(raw), cudaMemcpyDeviceToHost, s));
    if (!sci) CUDA_TRY(cudaMemcpyAsync(&leaves, a->dev.counters, sizeof(leaves), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    auto unorder = [](unsigned long long o) {
        const unsigned long long b = (o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o;
        double d;
        std::memcpy(&d, &b, 8);
        return d;
    };
    double mx, sum;
    std::memcpy(&mx, &raw[0], 8);
    std::memcpy(&sum, &raw[1], 8);
    const double count = (double)(leaves ? leaves : 1u) * 512.0 * (double)n;
    stats[0] = mx;
    stats[1] = std::sqrt(sum / count);
    stats[2] = unorder(raw[2]);
    stats[3] = unorder(raw[3]);
    return VBT_STATUS_OK;
}

int vbt_selftest_key_division(uint32_t b_max, uint64_t* result, int device)
{
    if (!result) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (b_max < 2u || b_max > 65535u) return fail(VBT_STATUS_INVALID_ARGUMENT, "b_max must lie in [2, 65535]");
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        return fail(VBT_STATUS_CUDA, "no CUDA device");
    if (device < 0 || device >= dev_count) return fail(VBT_STATUS_INVALID_ARGUMENT, "device out of range");
    DeviceGuard guard(device);
    unsigned long long* d = nullptr;
    CUDA_TRY(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
    const unsigned long long init[2] = {0ull, ~0ull};
    cudaError_t e = cudaMemcpy(d, init, sizeof(init), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        launch_key_division_check(b_max, d, nullptr);
        e = cudaGetLastError();
    }
    unsigned long long h[2] = {0ull, 0ull};
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(VBT_STATUS_CUDA, std::string("key division check: ") + cudaGetErrorString(e));
    result[0] = h[0];
    result[1] = h[1];
    return VBT_STATUS_OK;
}

int vbt_decode_control_values(const uint8_t* d_stream, uint32_t bytes, uint32_t codec, uint32_t cc, uint32_t bins,
                              uint32_t kf, int align, int total, const uint32_t* ci, const int32_t* fr, uint64_t n,
                              float* out, int32_t* status, void* stream)
{
    if (n && (!ci || !fr || !out)) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (n && !d_stream && bytes) return fail(VBT_STATUS_INVALID_ARGUMENT, "null stream");
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        return fail(VBT_STATUS_CUDA, "no usable CUDA device for the VBT decode path");
    launch_checked_decode(d_stream, bytes, codec, cc, bins, kf, align, total, ci, fr, n, out, status,
                          static_cast<cudaStream_t>(stream));
    return check_launch("checked_decode_kernel");
}

}  // extern "C"
