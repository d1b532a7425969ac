"""vbt_b200 -- B200-native (sm_100a) compressed-domain temporal decode of VBTPACK4 assets.

This module is a thin ctypes binding of the C-ABI in include/vbt_b200.h (libvbt_b200.so,
built in-tree by vbt_b200/build.py).  The decode work runs only in the CUDA kernels of that
library; there is no CPU execution path.  Importing this module fails loudly when the library
is missing; decode calls fail with VbtError(status=VBT_STATUS_CUDA) without a usable GPU.

Device buffers are passed as torch CUDA tensors (for their device pointers and streams only) or
as raw integer device addresses.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvbt_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"vbt_b200: {LIB_PATH} is missing; build it with `python vbt_b200/build.py`")

_lib = C.CDLL(LIB_PATH)

STATUS = {
    0: "OK", 1: "LEAF_TOO_SMALL", 2: "PREFIX_MISSING", 3: "LEAF_SHORT", 4: "SHELL_OCC_OOB",
    5: "SHELL_GROUP_PREFIX", 6: "SHELL_NO_ACTIVE", 7: "SHELL_RESIDUAL_OOB", 8: "SHELL_TRAILING",
    9: "CONTROL_INDEX", 10: "STREAM_OOB", 11: "DECODE_OOB", 12: "KEY_RANGE_OOB", 13: "KEY_INDEX",
    30: "WAIT_TIMEOUT", 40: "INVALID_ARGUMENT", 41: "FILE", 42: "CUDA", 43: "LIMIT", 44: "UNSUPPORTED",
}


class VbtHeader(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("version", "width", "height", "depth", "frames", "leaf_size",
                                          "coarse_resolution", "max_coarse_keep", "leaf_count", "profile_type",
                                          "coarse_ac_scale_count")]


class VbtAssetInfo(C.Structure):
    _fields_ = [("header", VbtHeader), ("leaf_count_x", C.c_uint32), ("leaf_count_y", C.c_uint32),
                ("leaf_count_z", C.c_uint32), ("active_leaf_count", C.c_uint32), ("payload_words", C.c_uint64),
                ("device_bytes", C.c_uint64), ("device", C.c_int)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget_bytes", C.c_uint64), ("host_staging_bytes", C.c_uint64),
                ("slots", C.c_uint32), ("max_batch_queries", C.c_uint32), ("plain", C.c_uint32),
                ("separate_kinds", C.c_uint32)]


class Request(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("asset", C.c_uint32), ("points", C.c_void_p), ("n_points", C.c_uint64),
                ("z", C.c_uint32), ("t0", C.c_int32), ("t1", C.c_int32), ("frames", C.c_void_p),
                ("n_frames", C.c_uint32), ("host_out", C.c_void_p)]


class SampleParams(C.Structure):
    """vbt_sample_params: the sampler's settings besides the asset's geometry."""
    _fields_ = [("step_count", C.c_uint32), ("frame_index", C.c_int32), ("bbox_min", C.c_float * 3),
                ("render_mode", C.c_uint32), ("voxel_size", C.c_float), ("background_value", C.c_float),
                ("surface_iso", C.c_float), ("surface_epsilon_voxels", C.c_float), ("surface_normal_step", C.c_float),
                ("max_step_voxels", C.c_float), ("surface_model", C.c_uint32), ("floor_height", C.c_float),
                ("shadow_steps", C.c_uint32), ("up_axis", C.c_uint32)]


class KeyframeProfile(C.Structure):
    """vbt_keyframe_profile: the encoder's DensityTemporalProfile and background threshold.  The
    defaults are the reference encoder's (src/render_temporal_kf_probe_main.cpp:51-58, :477)."""
    _fields_ = [("eps_abs", C.c_float), ("eps_rel", C.c_float), ("gamma_delta", C.c_float),
                ("render_cutoff", C.c_float), ("cutoff_band", C.c_float), ("cutoff_temporal_protect", C.c_uint32),
                ("iso_surface_protect", C.c_uint32), ("iso_value", C.c_float), ("iso_band", C.c_float),
                ("bg_threshold", C.c_double)]

    def __init__(self, **kw):
        d = dict(eps_abs=1e-5, eps_rel=0.02, gamma_delta=0.2, render_cutoff=0.0003, cutoff_band=0.0001,
                 cutoff_temporal_protect=1, iso_surface_protect=0, iso_value=0.0, iso_band=0.0)
        d.update(kw)
        if "bg_threshold" not in kw:   # bgZeroRatio (0.3) * cutoff, formed in float as the encoder does
            c = C.c_float(d["render_cutoff"]).value
            d["bg_threshold"] = float(C.c_float(C.c_float(0.3).value * c).value) if c > 0 else -1.0
        super().__init__(**d)


class KeyframeTotals(C.Structure):
    _fields_ = [("total_keys", C.c_uint64), ("protected_series", C.c_uint64), ("background_series", C.c_uint64),
                ("max_keys", C.c_uint32), ("pad", C.c_uint32), ("err2", C.c_double)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("bad_leaf", C.c_uint32), ("result_floats", C.c_uint64),
                ("device_result", C.c_void_p), ("submit_ms", C.c_double), ("start_ms", C.c_double),
                ("done_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("requests_done", C.c_uint64), ("points_done", C.c_uint64), ("voxels_done", C.c_uint64),
                ("launches", C.c_uint64), ("units", C.c_uint64), ("arena_peak_bytes", C.c_uint64),
                ("arena_bytes", C.c_uint64), ("resident_asset_bytes", C.c_uint64), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("max_ms", C.c_double), ("busy_ms", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("variant", C.c_uint32), ("frames_per_launch", C.c_uint32), ("grid", C.c_int),
                ("ms_per_frame", C.c_float), ("ms_per_frame_default", C.c_float)]


REQ_POINTS, REQ_SLICE, REQ_FRAMES = 1, 2, 3

_vp, _u32p, _i32p, _f32p = C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_int32), C.c_void_p
_sig = {
    "vbt_status_string": ([C.c_int], C.c_char_p),
    "vbt_last_error": ([], C.c_char_p),
    "vbt_device_count": ([], C.c_int),
    "vbt_validate_file_image": ([_vp, C.c_uint64, C.POINTER(VbtHeader)], C.c_int),
    "vbt_asset_open": ([C.c_char_p, C.c_int, C.POINTER(_vp)], C.c_int),
    "vbt_asset_create": ([_vp, C.c_uint64, C.c_int, C.POINTER(_vp)], C.c_int),
    "vbt_asset_destroy": ([_vp], C.c_int),
    "vbt_asset_upload": ([_vp, _vp, C.c_uint64, _vp], C.c_int),
    "vbt_asset_get_info": ([_vp, C.POINTER(VbtAssetInfo)], C.c_int),
    "vbt_build_page_table": ([_vp, _vp], C.c_int),
    "vbt_page_table_device": ([_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)], C.c_int),
    "vbt_get_page_table": ([_vp, _vp, _u32p], C.c_int),
    "vbt_get_leaf_table": ([_vp, _vp], C.c_int),
    "vbt_decode_cache": ([_vp, _i32p, C.c_int, _vp, C.c_uint64, C.c_int, _vp], C.c_int),
    "vbt_decode_cache_plain": ([_vp, C.c_int, _vp, _vp], C.c_int),
    "vbt_decode_frames": ([_vp, _i32p, C.c_int, _vp, C.c_int, _vp], C.c_int),
    "vbt_query_points": ([_vp, _vp, C.c_uint64, _vp, _vp], C.c_int),
    "vbt_query_slice": ([_vp, C.c_uint32, C.c_int, C.c_int, _vp, _vp], C.c_int),
    "vbt_asset_sync_status": ([_vp, _vp, _u32p], C.c_int),
    "vbt_query_points_host": ([_vp, _vp, C.c_uint64, _vp, _vp], C.c_int),
    "vbt_decode_frames_host": ([_vp, _i32p, C.c_int, _vp, _vp], C.c_int),
    "vbt_decode_control_values": ([_vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                                   C.c_int, _vp, _vp, C.c_uint64, _vp, _vp, _vp], C.c_int),
    "vbt_build_page_table_noalloc": ([_vp, _vp, C.c_uint64, C.c_uint32, C.c_uint32, _vp, _vp, _vp, _vp], C.c_int),
    "vbt_decode_window": ([_vp, C.c_int, C.c_int, _vp, C.c_uint64, _vp], C.c_int),
    "vbt_selftest_key_division": ([C.c_uint32, C.POINTER(C.c_uint64), C.c_int], C.c_int),
    "vbt_pack_payload": ([_vp, _vp, C.c_uint32, _vp, _vp, C.c_uint64, C.POINTER(C.c_uint64), _vp], C.c_int),
    "vbt_smoke_sample_rays": ([_vp, C.POINTER(SampleParams), _vp, C.c_uint32, _vp, _vp], C.c_int),
    "vbt_pack_leaves": ([_vp, C.c_uint32, _vp, _vp, C.c_uint64, _vp, _vp, C.c_uint64, _vp, C.c_uint64, _vp, _vp,
                         C.c_uint64, C.POINTER(C.c_uint64), _vp], C.c_int),
    "vbt_detect_keyframes": ([_vp, C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64, C.POINTER(KeyframeProfile), _vp,
                              _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "vbt_coarse_fit": ([_vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, _vp, C.c_uint32,
                        C.POINTER(KeyframeProfile), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "vbt_fine6_fit": ([_vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, _vp, C.c_uint32,
                       C.POINTER(KeyframeProfile), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "vbt_shell_fit": ([_vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, _vp, C.c_uint32,
                       C.POINTER(KeyframeProfile), _vp, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                       _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "vbt_route_density": ([_vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, _vp, C.c_uint32,
                           _vp, _vp, C.c_double, C.c_double, C.c_double, _vp, _vp], C.c_int),
    "vbt_selftest_keyframe_division": ([C.c_uint32, C.POINTER(C.c_uint64), C.c_int], C.c_int),
    "vbt_sample_rays": ([_vp, _vp, C.POINTER(SampleParams), _vp, C.c_uint32, _vp, _vp], C.c_int),
    "vbt_decode_control_cache": ([_vp, C.POINTER(C.c_int), C.c_int, _vp, C.c_uint64, _vp], C.c_int),
    "vbt_window_error": ([_vp, C.c_int, C.c_int, _vp, C.c_uint64, C.POINTER(C.c_double), _vp], C.c_int),
    "vbt_autotune_cache": ([_vp, C.c_int, _vp, C.c_uint64, C.POINTER(Tuning), _vp], C.c_int),
    "vbt_set_tuning": ([_vp, C.POINTER(Tuning)], C.c_int),
    "vbt_get_tuning": ([_vp, C.POINTER(Tuning)], C.c_int),
    "vbt_decode_cache_timeline": ([_vp, C.c_int, C.c_int, _vp, C.c_uint64, C.c_int, _vp], C.c_int),
    "vbt_server_create": ([C.POINTER(ServerConfig), C.POINTER(_vp)], C.c_int),
    "vbt_server_add_asset": ([_vp, _vp, _u32p], C.c_int),
    "vbt_serve_submit": ([_vp, C.POINTER(Request), C.POINTER(C.c_uint64)], C.c_int),
    "vbt_serve_poll": ([_vp, C.c_uint64, C.POINTER(C.c_int), C.POINTER(RequestResult)], C.c_int),
    "vbt_serve_wait": ([_vp, C.c_uint64, C.POINTER(RequestResult)], C.c_int),
    "vbt_serve_release": ([_vp, C.c_uint64], C.c_int),
    "vbt_server_get_stats": ([_vp, C.POINTER(ServerStats)], C.c_int),
    "vbt_server_reset_stats": ([_vp], C.c_int),
    "vbt_server_destroy": ([_vp], C.c_int),
}
for _name, (_args, _res) in _sig.items():
    _f = getattr(_lib, _name)
    _f.argtypes = _args
    _f.restype = _res

EXPORTS = tuple(_sig)


class VbtError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.message = message


def _check(status):
    if status != 0:
        raise VbtError(status, _lib.vbt_last_error().decode(errors="replace"))


def lib():
    return _lib


def device_count():
    return _lib.vbt_device_count()


def status_string(status):
    return _lib.vbt_status_string(status).decode()


def _addr(x):
    """Device address of a torch tensor or an int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return x.data_ptr()


def _stream(stream):
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.cuda.current_stream().cuda_stream
        except Exception:
            pass
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def validate_file_image(data):
    h = VbtHeader()
    buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
    _check(_lib.vbt_validate_file_image(C.cast(buf, _vp), len(data), C.byref(h)))
    return h


class Asset:
    """A VBTPACK4 asset resident on one GPU (offsets, payload, leaf table, page table)."""

    def __init__(self, path=None, data=None, device=0):
        self._h = _vp()
        if path is not None:
            _check(_lib.vbt_asset_open(os.fspath(path).encode(), device, C.byref(self._h)))
        elif hasattr(data, "data_ptr") or hasattr(data, "ctypes"):   # a host torch tensor or numpy array
            ptr = data.data_ptr() if hasattr(data, "data_ptr") else data.ctypes.data
            n = data.numel() * data.element_size() if hasattr(data, "data_ptr") else data.nbytes
            _check(_lib.vbt_asset_create(C.c_void_p(ptr), n, device, C.byref(self._h)))
        else:
            buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
            _check(_lib.vbt_asset_create(C.cast(buf, _vp), len(data), device, C.byref(self._h)))
        self.refresh_info()

    def refresh_info(self):
        info = VbtAssetInfo()
        _check(_lib.vbt_asset_get_info(self._h, C.byref(info)))
        self.info = info
        h = info.header
        self.dims = (h.width, h.height, h.depth)
        self.frames = h.frames
        self.leaf_count = h.leaf_count
        self.profile = h.profile_type
        self.active_count = info.active_leaf_count
        self.device = info.device
        return info

    def close(self):
        if self._h:
            _lib.vbt_asset_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def upload(self, host_image, stream=None):
        """Re-upload a file image (pinned torch uint8 tensor or numpy array) into this asset."""
        ptr = host_image.data_ptr() if hasattr(host_image, "data_ptr") else host_image.ctypes.data
        n = host_image.numel() if hasattr(host_image, "numel") else host_image.nbytes
        _check(_lib.vbt_asset_upload(self._h, ptr, n, _stream(stream)))

    # kernel (a)
    def build_page_table(self, stream=None):
        _check(_lib.vbt_build_page_table(self._h, _stream(stream)))

    def page_table_device(self):
        c, l, n = _vp(), _vp(), _vp()
        _check(_lib.vbt_page_table_device(self._h, C.byref(c), C.byref(l), C.byref(n)))
        return c.value, l.value, n.value

    def page_table(self):
        import numpy as np
        compact = np.zeros(self.leaf_count, np.uint32)
        n = C.c_uint32()
        _check(_lib.vbt_get_page_table(self._h, compact.ctypes.data, C.byref(n)))
        return compact, n.value

    def leaf_table(self):
        import numpy as np
        rows = np.zeros((self.leaf_count, 8), np.uint32)
        _check(_lib.vbt_get_leaf_table(self._h, rows.ctypes.data))
        return rows

    # kernel (b)
    def decode_cache(self, frames, out, frame_stride=None, grid=0, stream=None):
        fr = (C.c_int32 * len(frames))(*frames)
        if frame_stride is None:
            frame_stride = self.active_count * 512
        _check(_lib.vbt_decode_cache(self._h, fr, len(frames), _addr(out), frame_stride, grid, _stream(stream)))

    def decode_control_cache(self, frames, out, frame_stride=None, stream=None):
        """The Studio's 576-slot control cache of `frames` over the current page table's active
        leaves: out[f * frame_stride + rank * 576 + slot]."""
        fr = (C.c_int * len(frames))(*frames)
        stride = self.active_count * 576 if frame_stride is None else frame_stride
        _check(_lib.vbt_decode_control_cache(self._h, fr, len(frames), _addr(out), stride, _stream(stream)))

    def sample_rays(self, controls, params, rays, out, stream=None):
        """Ray sampling from the control cache `controls` of frame params.frame_index: rays [n, 8]
        (origin, t_min, direction, t_max) and out [n, 8] float32 device tensors."""
        n = rays.shape[0]
        _check(_lib.vbt_sample_rays(self._h, _addr(controls), C.byref(params), _addr(rays), n, _addr(out),
                                    _stream(stream)))

    def smoke_sample_rays(self, params, rays, out, stream=None):
        """The render tree's smoke sampler (vbt_smoke_sample.comp): rays [n, 8] float32 device tensor
        -> out [n] float32, the sum of params.step_count density samples per ray, decoded straight
        from the payload."""
        n = rays.numel() // 8
        _check(_lib.vbt_smoke_sample_rays(self._h, C.byref(params), _addr(rays), n, _addr(out), _stream(stream)))

    def decode_window(self, t0, n, out, frame_stride=None, stream=None):
        """(d) window decode on the tensor cores of frames [t0, t0 + n) into `out` in the cache
        layout: scientific assets n <= 64, every leaf; render assets n <= 64 as 16-frame
        windows, the active leaves of the current page table (build it first)."""
        stride = self.leaf_count * 512 if frame_stride is None else frame_stride
        _check(_lib.vbt_decode_window(self._h, t0, n, _addr(out), stride, _stream(stream)))

    def window_error(self, t0, n, values, frame_stride=None, stream=None):
        """FP64 oracle error of a cache of frames [t0, t0 + n) (scientific: every leaf; render:
        the active leaves of the current page table): (max_abs, rms, oracle_min, oracle_max)."""
        stride = self.leaf_count * 512 if frame_stride is None else frame_stride
        st = (C.c_double * 4)()
        _check(_lib.vbt_window_error(self._h, t0, n, _addr(values), stride, st, _stream(stream)))
        return tuple(st)

    def autotune(self, nframes, out, frame_stride=None, stream=None):
        """Time the cache-timeline launch shapes on `out` and keep the fastest (returns Tuning)."""
        t = Tuning()
        stride = self.active_count * 512 if frame_stride is None else frame_stride
        _check(_lib.vbt_autotune_cache(self._h, nframes, _addr(out), stride, C.byref(t), _stream(stream)))
        return t

    def set_tuning(self, variant, frames_per_launch, grid=0):
        t = Tuning(variant, frames_per_launch, grid, 0.0, 0.0)
        _check(_lib.vbt_set_tuning(self._h, C.byref(t)))

    def tuning(self):
        t = Tuning()
        _check(_lib.vbt_get_tuning(self._h, C.byref(t)))
        return t

    def decode_cache_timeline(self, t0, n, out, frame_stride=None, graph=True, stream=None):
        """Page table + cache of frames [t0, t0 + n) with the asset's tuning; graph=True replays a
        CUDA graph captured on the first call for this (t0, n, out, stride)."""
        stride = self.active_count * 512 if frame_stride is None else frame_stride
        _check(_lib.vbt_decode_cache_timeline(self._h, t0, n, _addr(out), stride, int(graph), _stream(stream)))

    def decode_cache_plain(self, frame, out, stream=None):
        _check(_lib.vbt_decode_cache_plain(self._h, frame, _addr(out), _stream(stream)))

    def decode_frames(self, frames, out, grid=0, stream=None):
        fr = (C.c_int32 * len(frames))(*frames)
        _check(_lib.vbt_decode_frames(self._h, fr, len(frames), _addr(out), grid, _stream(stream)))

    # kernel (c)
    def query_points(self, xyzt, out, stream=None):
        n = xyzt.shape[0] if hasattr(xyzt, "shape") else 0
        _check(_lib.vbt_query_points(self._h, _addr(xyzt), n, _addr(out), _stream(stream)))

    def query_slice(self, z, t0, t1, out, stream=None):
        _check(_lib.vbt_query_slice(self._h, z, t0, t1, _addr(out), _stream(stream)))

    def sync_status(self, stream=None):
        bad = C.c_uint32()
        st = _lib.vbt_asset_sync_status(self._h, _stream(stream), C.byref(bad))
        if st != 0:
            raise VbtError(st, _lib.vbt_last_error().decode(errors="replace"))
        return True

    # host-buffer (end-to-end) calls
    def query_points_host(self, xyzt, out, stream=None):
        _check(_lib.vbt_query_points_host(self._h, xyzt.ctypes.data, xyzt.shape[0], out.ctypes.data,
                                          _stream(stream)))

    def decode_frames_host(self, frames, out, stream=None):
        fr = (C.c_int32 * len(frames))(*frames)
        _check(_lib.vbt_decode_frames_host(self._h, fr, len(frames), out.ctypes.data, _stream(stream)))


def pack_payload(blocks, block_offsets, offsets, payload, stream=None):
    """VBTPACK4 payload assembly on the GPU: blocks (uint8 device tensor), block_offsets (int64
    device tensor, n + 1 byte offsets) -> offsets (int32 device tensor, n + 1 word offsets) and
    payload (int32 device tensor); returns the payload size in words."""
    total = C.c_uint64()
    n = block_offsets.shape[0] - 1
    _check(_lib.vbt_pack_payload(_addr(blocks), _addr(block_offsets), n, _addr(offsets), _addr(payload),
                                 payload.numel() if payload is not None else 0, C.byref(total), _stream(stream)))
    return total.value


def pack_leaves(leaves, descriptors, bins, key_frames, key_values, occupancy, offsets, payload, stream=None):
    """VBTPACK4 leaves from their control streams on the GPU, straight into the payload.  leaves: a
    uint8 device tensor of 32-byte vbt_leaf_streams records; descriptors (int32, one per control
    row), bins (uint8, 8 per control row), key_frames (int16/uint16), key_values (float32),
    occupancy (uint8, 80 per Mode2 section, may be None); offsets (int32, n + 1) and payload
    (int32) receive the result.  Returns the payload size in words."""
    total = C.c_uint64()
    n = leaves.numel() // 32
    rows = lambda t, per=1: 0 if t is None else t.numel() // per  # noqa: E731
    _check(_lib.vbt_pack_leaves(_addr(leaves), n, _addr(descriptors), _addr(bins),
                                min(rows(descriptors), rows(bins, 8)), _addr(key_frames), _addr(key_values),
                                min(rows(key_frames), rows(key_values)), _addr(occupancy),
                                rows(occupancy, 80), _addr(offsets), _addr(payload),
                                payload.numel() if payload is not None else 0, C.byref(total), _stream(stream)))
    return total.value


def detect_keyframes(values, profile, key_mask, key_count, flags, recon=None, err2=None, totals=None,
                     series=None, time_fastest=False, stream=None):
    """The encoder's per-voxel keyframe pass on the GPU.  values: a float32 device tensor, frame-major
    [frames, >= series] or, with time_fastest, [series, >= frames] (rows may be padded); `series`
    defaults to all of them.  Outputs: key_mask [ceil(frames / 32), series] int32, key_count
    [series] int32, flags [series] uint8, and optionally recon (the reconstruction, in values'
    layout), err2 [series] float64 and totals (a 40-byte device buffer read back by
    keyframe_totals)."""
    if time_fastest:
        rows, frames = values.shape
        ss, fs = values.stride()
        n = rows if series is None else int(series)
    else:
        frames, cols = values.shape
        fs, ss = values.stride()
        n = cols if series is None else int(series)
    if recon is not None and tuple(recon.stride()) != tuple(values.stride()):
        raise ValueError("recon must have the layout of values")
    _check(_lib.vbt_detect_keyframes(_addr(values), n, frames, fs, ss, C.byref(profile), _addr(key_mask),
                                     _addr(key_count), _addr(flags), _addr(recon), _addr(err2), _addr(totals),
                                     _stream(stream)))


def coarse_fit(recon, dims, leaves, profile, desc, bins, key_frames, key_values, key_count, required,
               grid=None, stream=None):
    """The encoder's coarse control fitting on the GPU over the frame-major reconstruction recon
    [frames, >= X*Y*Z] (float32 device tensor) of a volume dims = (X, Y, Z), for the leaf indices in
    leaves (int32 device tensor).  Outputs (device tensors): desc [n, 64] int32, bins [n, 64, 8]
    uint8, key_frames / key_values [n, 64 * frames] int16 / float32, key_count [n] int32, required
    [n] uint8, and optionally grid [n, 64, frames] float32."""
    frames, stride = recon.shape
    X, Y, Z = dims
    _check(_lib.vbt_coarse_fit(_addr(recon), X, Y, Z, frames, recon.stride(0), _addr(leaves), leaves.numel(),
                               C.byref(profile), _addr(desc), _addr(bins), _addr(key_frames), _addr(key_values),
                               _addr(key_count), _addr(required), _addr(grid), _stream(stream)))


def fine6_fit(recon, dims, leaves, profile, coarse_grid, desc, bins, key_frames, key_values, key_count, required,
              grid=None, stream=None):
    """The encoder's FINE6 residual fitting on the GPU: as coarse_fit for the 6^3 controls at
    controlCoords(6), each series the sampled reconstruction minus coarse_grid ([n, 64, frames],
    coarse_fit's grid of the same leaves) sampled at the same position.  Outputs desc [n, 216],
    bins [n, 216, 8], key_frames / key_values [n, 216 * frames], key_count [n], required [n] and
    optionally grid [n, 216, frames]."""
    frames = recon.shape[0]
    X, Y, Z = dims
    _check(_lib.vbt_fine6_fit(_addr(recon), X, Y, Z, frames, recon.stride(0), _addr(leaves), leaves.numel(),
                              C.byref(profile), _addr(coarse_grid), _addr(desc), _addr(bins), _addr(key_frames),
                              _addr(key_values), _addr(key_count), _addr(required), _addr(grid), _stream(stream)))


def shell_fit(recon, dims, leaves, profile, coarse_grid, levelset, surface_band, guard_band, temporal_band, shell_cut,
              occupancy, desc, bins, key_frames, key_values, key_count, active, required, stream=None):
    """The encoder's Mode2 shell stage on the GPU for the listed leaves: occupancy [n, 80] uint8, desc
    [n, 512], bins [n, 512, 8], key_frames / key_values [n, 512 * frames], key_count [n], active [n]
    (shell voxels) and required [n]."""
    frames = recon.shape[0]
    X, Y, Z = dims
    _check(_lib.vbt_shell_fit(_addr(recon), X, Y, Z, frames, recon.stride(0), _addr(leaves), leaves.numel(),
                              C.byref(profile), _addr(coarse_grid), int(levelset), surface_band, guard_band,
                              temporal_band, shell_cut, _addr(occupancy), _addr(desc), _addr(bins), _addr(key_frames),
                              _addr(key_values), _addr(key_count), _addr(active), _addr(required), _stream(stream)))


def route_density(raw, dims, leaves, coarse_grid, fine_grid, peak, visible_lo, visible_hi, mode, stream=None):
    """The encoder's density route per listed leaf (mode [n] uint8: 3 FINE6, 1 GRID4) from the raw
    field raw [frames, >= X*Y*Z] and the fitted coarse and fine grids."""
    frames = raw.shape[0]
    X, Y, Z = dims
    _check(_lib.vbt_route_density(_addr(raw), X, Y, Z, frames, raw.stride(0), _addr(leaves), leaves.numel(),
                                  _addr(coarse_grid), _addr(fine_grid), float(peak), float(visible_lo),
                                  float(visible_hi), _addr(mode), _stream(stream)))


def keyframe_totals(buf):
    """KeyframeTotals from the device buffer `detect_keyframes` filled (a uint8 tensor of 40 bytes)."""
    raw = bytes(buf.cpu().numpy().tobytes())
    return KeyframeTotals.from_buffer_copy(raw[:C.sizeof(KeyframeTotals)])


def selftest_keyframe_division(b_max=1024, device=0):
    """(mismatches, smallest failing b << 16 | a) of the keyframe pass's integer quotient
    a / b against IEEE division, over every 0 <= a <= b <= b_max."""
    r = (C.c_uint64 * 2)()
    _check(_lib.vbt_selftest_keyframe_division(b_max, r, device))
    return int(r[0]), int(r[1])


def selftest_key_division(b_max=65535, device=0):
    """(mismatches, smallest failing b << 16 | a) of the render decode's division-free interval
    quotient against IEEE division, over every 0 < a < b <= b_max."""
    r = (C.c_uint64 * 2)()
    _check(_lib.vbt_selftest_key_division(b_max, r, device))
    return int(r[0]), int(r[1])


def build_page_table_noalloc(d_offsets, d_payload, payload_words, leaf_count, profile_type, d_compact,
                             d_active_list, d_active_count, stream=None):
    """Page table from caller-owned device buffers; the library allocates nothing (see the C
    declaration in include/vbt_b200.h for the scratch array and its limit)."""
    _check(_lib.vbt_build_page_table_noalloc(_addr(d_offsets), _addr(d_payload), payload_words, leaf_count,
                                             profile_type, _addr(d_compact), _addr(d_active_list),
                                             _addr(d_active_count), _stream(stream)))


def decode_control_values(d_stream, stream_bytes, codec, control_count, bins, kf, total_frames, d_ci, d_frames, n,
                          d_out, d_status, align=True, stream=None):
    _check(_lib.vbt_decode_control_values(_addr(d_stream), stream_bytes, codec, control_count, bins, kf, int(align),
                                          total_frames, _addr(d_ci), _addr(d_frames), n, _addr(d_out),
                                          _addr(d_status), _stream(stream)))


class Server:
    """The serving loop (vbt_server_* in include/vbt_b200.h): resident assets, requests admitted
    by an HBM budget, the requests admitted together run as one mixed persistent launch (or, with
    separate_kinds, only point requests merged), launches overlapped on `slots` streams.

    Host buffers handed to submit_*() (numpy arrays) must stay alive until the request is done;
    the object keeps references to them until release()."""

    def __init__(self, hbm_budget_bytes=1 << 30, slots=4, max_batch_queries=0, plain=False, device=0,
                 host_staging_bytes=256 << 20, separate_kinds=False):
        cfg = ServerConfig(device, hbm_budget_bytes, host_staging_bytes, slots, max_batch_queries, int(plain),
                           int(separate_kinds))
        self._h = _vp()
        _check(_lib.vbt_server_create(C.byref(cfg), C.byref(self._h)))
        self._keep = {}

    def add_asset(self, asset):
        i = C.c_uint32()
        _check(_lib.vbt_server_add_asset(self._h, asset.handle, C.byref(i)))
        return i.value

    def _submit(self, req, keep):
        t = C.c_uint64()
        _check(_lib.vbt_serve_submit(self._h, C.byref(req), C.byref(t)))
        self._keep[t.value] = keep
        return t.value

    @staticmethod
    def _buf(x):
        """Address of a numpy array (host) or a torch tensor (host or device memory), or None."""
        if x is None:
            return None
        return x.data_ptr() if hasattr(x, "data_ptr") else x.ctypes.data

    def submit_points(self, asset_id, xyzt, host_out=None):
        """xyzt: contiguous uint32 [n, 4] in host memory (numpy, or a pinned torch tensor) or device
        memory (a CUDA torch tensor); host_out: float32 [n] likewise, or None to keep the result in
        device memory until release()."""
        req = Request(kind=REQ_POINTS, asset=asset_id, points=self._buf(xyzt), n_points=xyzt.shape[0],
                      host_out=self._buf(host_out))
        return self._submit(req, (xyzt, host_out))

    def submit_slice(self, asset_id, z, t0, t1, host_out=None):
        req = Request(kind=REQ_SLICE, asset=asset_id, z=z, t0=t0, t1=t1, host_out=self._buf(host_out))
        return self._submit(req, (host_out,))

    def submit_frames(self, asset_id, frames, host_out=None):
        fr = (C.c_int32 * len(frames))(*frames)
        req = Request(kind=REQ_FRAMES, asset=asset_id, frames=C.cast(fr, C.c_void_p), n_frames=len(frames),
                      host_out=self._buf(host_out))
        return self._submit(req, (fr, host_out))

    def poll(self, ticket):
        done = C.c_int()
        res = RequestResult()
        _check(_lib.vbt_serve_poll(self._h, ticket, C.byref(done), C.byref(res)))
        return bool(done.value), res

    def wait(self, ticket):
        res = RequestResult()
        _check(_lib.vbt_serve_wait(self._h, ticket, C.byref(res)))
        return res

    def release(self, ticket):
        _check(_lib.vbt_serve_release(self._h, ticket))
        self._keep.pop(ticket, None)

    def stats(self):
        st = ServerStats()
        _check(_lib.vbt_server_get_stats(self._h, C.byref(st)))
        return st

    def reset_stats(self):
        _check(_lib.vbt_server_reset_stats(self._h))

    def close(self):
        if self._h:
            _lib.vbt_server_destroy(self._h)
            self._h = _vp()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
