"""ctypes bindings for the parity checker (test infrastructure only).

``Oracle`` wraps liboracle.so, the C restatement of the reference decode path
(vbt_oracle.c).  ``Reference`` wraps oracle/_ref/libvbtref.so, the reference decoder
compiled from its own sources.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg use this module; the product (vbt_b200) never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libvbtref.so")
KFREF_SO = os.path.join(HERE, "_ref", "libkfref.so")

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
f32p = C.POINTER(C.c_float)


def _ptr(a, t):
    return a.ctypes.data_as(t)


class VoFile(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("version", "width", "height", "depth", "frames", "leaf_size",
                                          "coarse_res", "max_coarse_keep", "leaf_count", "profile_type",
                                          "scale_count")] + [
        ("scales", f32p), ("offsets", u32p), ("payload", u32p), ("payload_words", C.c_uint64)]


class VoStream(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("desc_off", "desc_bytes", "bin_off", "bin_bytes", "key_off",
                                          "key_bytes", "total")]


class VoHeader(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("mode", "coarse_codec", "fine_codec", "coarse_res", "fine_res")]


class VoSampleParams(C.Structure):
    """vo_sample_params (vbt_oracle.h); the same layout as vbt_sample_params (include/vbt_b200.h)."""
    _fields_ = [("step_count", C.c_uint32), ("frame_index", C.c_int32), ("bbox_min", C.c_float * 3),
                ("render_mode", C.c_uint32), ("voxel_size", C.c_float), ("background_value", C.c_float),
                ("surface_iso", C.c_float), ("surface_epsilon_voxels", C.c_float), ("surface_normal_step", C.c_float),
                ("max_step_voxels", C.c_float), ("surface_model", C.c_uint32), ("floor_height", C.c_float),
                ("shadow_steps", C.c_uint32), ("up_axis", C.c_uint32)]


class VoKeyframeProfile(C.Structure):
    """vo_keyframe_profile (vbt_oracle.h); the same layout as vbt_keyframe_profile (include/vbt_b200.h).
    Defaults are the reference encoder's (src/render_temporal_kf_probe_main.cpp:51-58, :477)."""
    _fields_ = [("eps_abs", C.c_float), ("eps_rel", C.c_float), ("gamma_delta", C.c_float),
                ("render_cutoff", C.c_float), ("cutoff_band", C.c_float), ("cutoff_temporal_protect", C.c_uint32),
                ("iso_surface_protect", C.c_uint32), ("iso_value", C.c_float), ("iso_band", C.c_float),
                ("bg_threshold", C.c_double)]

    def __init__(self, **kw):
        d = dict(eps_abs=1e-5, eps_rel=0.02, gamma_delta=0.2, render_cutoff=0.0003, cutoff_band=0.0001,
                 cutoff_temporal_protect=1, iso_surface_protect=0, iso_value=0.0, iso_band=0.0)
        d.update(kw)
        if "bg_threshold" not in kw:   # bgZeroRatio * cutoff in float, as the encoder forms it
            c = np.float32(d["render_cutoff"])
            d["bg_threshold"] = float(np.float32(0.3) * c) if c > 0 else -1.0
        super().__init__(**d)


class VoLeafView(C.Structure):
    _fields_ = [("header", VoHeader), ("coarse_kf", C.c_uint32), ("fine_kf", C.c_uint32),
                ("coarse_off", C.c_uint32), ("fine_off", C.c_uint32), ("total", C.c_uint32),
                ("coarse", VoStream), ("fine", VoStream), ("shell_active", C.c_uint32),
                ("shell_residual_off", C.c_uint32), ("shell_residual_bytes", C.c_uint32)]


def reference_tree():
    """The VBT source tree the _ref targets compile (VBT_REFERENCE_TREE, default: a "reference"
    directory beside this repository), or None where it is absent."""
    ref = os.environ.get("VBT_REFERENCE_TREE", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
    return ref if os.path.isdir(os.path.join(ref, "src")) else None


def build(ref=False):
    """Build liboracle.so (and, when the reference tree exists, oracle/_ref)."""
    tree = reference_tree() if ref else None
    targets = ["oracle"] + (["ref", "REF=" + tree] if tree else [])
    subprocess.check_call(["make", "-s", "-C", HERE, "-j8"] + targets)


def pack_payload(blocks):
    """The payload half of writeRenderTemporalProbeFile (src/render_temporal_kf_probe_main.cpp:
    2561-2585): offsetsWords[i] = payload bytes so far / 4, each leaf block padded with zero bytes
    to a multiple of 4, offsetsWords[n] = payload words.  blocks: list of bytes."""
    offsets = np.zeros(len(blocks) + 1, np.uint32)
    pool = bytearray()
    for i, b in enumerate(blocks):
        offsets[i] = len(pool) // 4
        pool += bytes(b) + b"\0" * ((4 - len(b) % 4) % 4)
    offsets[-1] = len(pool) // 4
    return offsets, np.frombuffer(bytes(pool), np.uint32).copy()


class Oracle:
    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build()
        L = self.lib = C.CDLL(ORACLE_SO)
        L.vo_load_file.argtypes = [C.c_char_p, C.POINTER(VoFile), C.c_char_p, C.c_size_t]
        L.vo_load_image.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(VoFile), C.c_char_p, C.c_size_t]
        L.vo_free_file.argtypes = [C.POINTER(VoFile)]
        L.vo_decode_frame.argtypes = [C.POINTER(VoFile), C.c_int, f32p, C.c_int, u32p]
        L.vo_build_page_table.argtypes = [C.POINTER(VoFile), u32p]
        L.vo_build_page_table.restype = C.c_uint32
        L.vo_decode_cache.argtypes = [C.POINTER(VoFile), C.c_int, u32p, f32p, C.c_int]
        L.vo_query_points.argtypes = [C.POINTER(VoFile), u32p, C.c_uint64, f32p, C.c_int]
        L.vo_sci_frame.argtypes = [C.POINTER(VoFile), C.c_uint32, f32p, C.c_int]
        L.vo_sci_query_points.argtypes = [C.POINTER(VoFile), u32p, C.c_uint64, f32p, C.c_int]
        L.vo_control_cache.argtypes = [C.POINTER(VoFile), C.c_int, u32p, f32p]
        L.vo_sample_rays.argtypes = [C.POINTER(VoFile), f32p, u32p, C.POINTER(VoSampleParams), f32p, C.c_uint32, f32p]
        L.vo_smoke_sample_rays.argtypes = [C.POINTER(VoFile), C.POINTER(VoSampleParams), f32p, C.c_uint32, f32p]
        L.vo_decode_control.argtypes = [u8p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                                        C.c_int, C.c_uint32, C.c_int, f32p]
        L.vo_decode_shell_voxel.argtypes = [u8p, C.POINTER(VoLeafView), C.c_int, C.c_uint32, C.c_int, f32p]
        L.vo_parse_leaf.argtypes = [u8p, C.c_size_t, C.c_int, C.POINTER(VoLeafView)]
        L.vo_decode_leaf_frame.argtypes = [u8p, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, f32p]
        L.vo_half_to_float.argtypes = [C.c_uint16]
        L.vo_half_to_float.restype = C.c_float
        L.vo_float_to_half.argtypes = [C.c_float]
        L.vo_float_to_half.restype = C.c_uint16
        L.vo_dct_basis.restype = C.c_float
        L.vo_dct_basis_f64.restype = C.c_double
        i32p = C.POINTER(C.c_int)
        L.vo_detect_keyframes.argtypes = [f32p, C.c_int, C.POINTER(VoKeyframeProfile), i32p, i32p]
        L.vo_reconstruct.argtypes = [f32p, C.c_int, i32p, C.c_int, f32p]
        L.vo_fine6_fit.argtypes = [f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(VoKeyframeProfile), f32p, u32p,
                                   u8p, C.POINTER(C.c_uint16), f32p, C.c_int, C.POINTER(C.c_int), f32p]
        L.vo_shell_fit.argtypes = [f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(VoKeyframeProfile), f32p,
                                   C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, u8p, u32p, u8p,
                                   C.POINTER(C.c_uint16), f32p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.vo_float_to_half_n.argtypes = [f32p, C.c_uint64, C.POINTER(C.c_uint16)]
        L.vo_coarse_fit.argtypes = [f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(VoKeyframeProfile), u32p, u8p,
                                    C.POINTER(C.c_uint16), f32p, C.c_int, C.POINTER(C.c_int), f32p]
        L.vo_keyframe_pass.argtypes = [f32p, C.c_uint64, C.c_int, C.c_uint64, C.POINTER(VoKeyframeProfile), u32p,
                                       u32p, u8p, f32p, C.POINTER(C.c_double), C.c_int]

    def detect_keyframes(self, series, profile):
        """(keys, used_protect) of detectDensityKeyFrames on one series."""
        v = np.ascontiguousarray(series, np.float32)
        keys = np.zeros(max(1, v.size), np.int32)
        used = C.c_int()
        k = self.lib.vo_detect_keyframes(_ptr(v, f32p), v.size, C.byref(profile), _ptr(keys, C.POINTER(C.c_int)),
                                         C.byref(used))
        return keys[:k].copy(), bool(used.value)

    def reconstruct(self, series, keys):
        v = np.ascontiguousarray(series, np.float32)
        k = np.ascontiguousarray(keys, np.int32)
        out = np.zeros(v.size, np.float32)
        self.lib.vo_reconstruct(_ptr(v, f32p), v.size, _ptr(k, C.POINTER(C.c_int)), k.size, _ptr(out, f32p))
        return out

    def fine6_fit(self, leaf_recon, extent, profile, coarse_grid):
        """The FINE6 residual fitting of one leaf over its fitted coarse grid [64, T] (coarse_fit's
        grid): dict of desc [216], bins [216, 8], key_frames, key_values, required_max_local, grid."""
        lt = np.ascontiguousarray(leaf_recon, np.float32).reshape(512, -1)
        T = lt.shape[1]
        cg = np.ascontiguousarray(coarse_grid, np.float32)
        cap = 216 * max(T, 1)
        desc = np.zeros(216, np.uint32)
        bins = np.zeros((216, 8), np.uint8)
        kf = np.zeros(cap, np.uint16)
        kv = np.zeros(cap, np.float32)
        grid = np.zeros((216, T), np.float32)
        req = C.c_int()
        n = self.lib.vo_fine6_fit(_ptr(lt, f32p), T, *extent, C.byref(profile), _ptr(cg, f32p), _ptr(desc, u32p),
                                  _ptr(bins, u8p), _ptr(kf, C.POINTER(C.c_uint16)), _ptr(kv, f32p), cap, C.byref(req),
                                  _ptr(grid, f32p))
        return dict(desc=desc, bins=bins, key_frames=kf[:n].copy(), key_values=kv[:n].copy(),
                    required_max_local=req.value, grid=grid)

    def shell_fit(self, leaf_recon, extent, profile, coarse_grid, levelset, surface_band, guard_band, temporal_band,
                  shell_cut):
        """The Mode2 shell stage of one leaf: dict of occupancy (80 bytes), desc [active], bins
        [active, 8], key_frames, key_values, active, required_max_local."""
        lt = np.ascontiguousarray(leaf_recon, np.float32).reshape(512, -1)
        T = lt.shape[1]
        cg = np.ascontiguousarray(coarse_grid, np.float32)
        cap = 512 * max(T, 1)
        occ = np.zeros(80, np.uint8)
        desc = np.zeros(512, np.uint32)
        bins = np.zeros((512, 8), np.uint8)
        kf = np.zeros(cap, np.uint16)
        kv = np.zeros(cap, np.float32)
        act, req = C.c_int(), C.c_int()
        n = self.lib.vo_shell_fit(_ptr(lt, f32p), T, *extent, C.byref(profile), _ptr(cg, f32p), int(levelset),
                                  surface_band, guard_band, temporal_band, shell_cut, _ptr(occ, u8p), _ptr(desc, u32p),
                                  _ptr(bins, u8p), _ptr(kf, C.POINTER(C.c_uint16)), _ptr(kv, f32p), cap, C.byref(act),
                                  C.byref(req))
        a = act.value
        return dict(occupancy=occ, desc=desc[:a].copy(), bins=bins[:a].copy(), key_frames=kf[:n].copy(),
                    key_values=kv[:n].copy(), active=a, required_max_local=req.value)

    def float_to_half(self, values):
        """renderTemporalFloatToHalfBits of every value (uint16 array)."""
        v = np.ascontiguousarray(values, np.float32).reshape(-1)
        out = np.zeros(v.size, np.uint16)
        self.lib.vo_float_to_half_n(_ptr(v, f32p), v.size, _ptr(out, C.POINTER(C.c_uint16)))
        return out

    def coarse_fit(self, leaf_recon, extent, profile):
        """The encoder's coarse control fitting of one leaf: leaf_recon [512, T] (voxel (lz*8+ly)*8+lx,
        frames fastest) -> dict of desc [64] u32, bins [64, 8] u8, key_frames, key_values,
        required_max_local and grid [64, T]."""
        return _coarse_fit(self.lib.vo_coarse_fit, leaf_recon, extent, profile)

    def keyframe_pass(self, frames, profile, threads=0):
        """The encoder's per-voxel pass over frames[T, S] (frame-major): dict of key_mask [W, S] u32,
        key_count [S] u32, flags [S] u8, recon [T, S] f32 and err2 [S] f64."""
        v = np.ascontiguousarray(frames, np.float32)
        T, S = v.shape
        W = (T + 31) // 32
        out = dict(key_mask=np.zeros((W, S), np.uint32), key_count=np.zeros(S, np.uint32),
                   flags=np.zeros(S, np.uint8), recon=np.zeros((T, S), np.float32), err2=np.zeros(S, np.float64))
        self.lib.vo_keyframe_pass(_ptr(v, f32p), S, T, S, C.byref(profile), _ptr(out["key_mask"], u32p),
                                  _ptr(out["key_count"], u32p), _ptr(out["flags"], u8p), _ptr(out["recon"], f32p),
                                  _ptr(out["err2"], C.POINTER(C.c_double)), threads if threads else os.cpu_count())
        return out

    def load(self, path=None, image=None):
        return OracleFile(self, path, image)

    def decode_control(self, stream, codec, cc, bins, kf, stream_bytes, total, ci, frame, align=True):
        s = np.ascontiguousarray(stream, np.uint8)
        out = C.c_float()
        st = self.lib.vo_decode_control(_ptr(s, u8p), codec, cc, bins, kf, stream_bytes, int(align), total, ci,
                                        frame, C.byref(out))
        return st, out.value

    def parse_leaf(self, leaf):
        b = np.ascontiguousarray(leaf, np.uint8)
        v = VoLeafView()
        st = self.lib.vo_parse_leaf(_ptr(b, u8p), b.size, 1, C.byref(v))
        return st, v

    def shell_voxel(self, leaf, total, voxel, frame):
        b = np.ascontiguousarray(leaf, np.uint8)
        st, v = self.parse_leaf(b)
        if st:
            return st, 0.0
        out = C.c_float()
        st = self.lib.vo_decode_shell_voxel(_ptr(b, u8p), C.byref(v), total, voxel, frame, C.byref(out))
        return st, out.value

    def decode_leaf(self, leaf, total, frame, w=8, h=8, d=8):
        b = np.ascontiguousarray(leaf, np.uint8)
        out = np.zeros(w * h * d, np.float32)
        st = self.lib.vo_decode_leaf_frame(_ptr(b, u8p), b.size, total, frame, w, h, d, _ptr(out, f32p))
        return st, out


class OracleFile:
    """A VBTPACK4 file in the oracle: from a path, or from a file image held in memory (bytes, a
    numpy array or a host torch tensor)."""

    def __init__(self, oracle, path=None, image=None):
        self.o = oracle
        self.f = VoFile()
        err = C.create_string_buffer(512)
        if path is not None:
            st = oracle.lib.vo_load_file(os.fspath(path).encode(), C.byref(self.f), err, 512)
        elif isinstance(image, (bytes, bytearray)):
            buf = (C.c_uint8 * len(image)).from_buffer_copy(image)
            st = oracle.lib.vo_load_image(C.cast(buf, C.c_void_p), len(image), C.byref(self.f), err, 512)
        else:
            ptr = image.data_ptr() if hasattr(image, "data_ptr") else image.ctypes.data
            n = image.numel() * image.element_size() if hasattr(image, "data_ptr") else image.nbytes
            st = oracle.lib.vo_load_image(C.c_void_p(ptr), n, C.byref(self.f), err, 512)
        if st != 0:
            raise RuntimeError(err.value.decode())
        self.dims = (self.f.width, self.f.height, self.f.depth)
        self.frames = self.f.frames
        self.leaf_count = self.f.leaf_count
        self.profile = self.f.profile_type

    def __del__(self):
        try:
            self.o.lib.vo_free_file(C.byref(self.f))
        except Exception:
            pass

    def offsets(self):
        return np.ctypeslib.as_array(self.f.offsets, (self.f.leaf_count + 1,)).copy()

    def payload(self):
        return np.ctypeslib.as_array(self.f.payload, (int(self.f.payload_words),)).copy()

    def frame(self, t, threads=0):
        X, Y, Z = self.dims
        out = np.zeros(Z * Y * X, np.float32)
        if self.profile == 2:
            self.o.lib.vo_sci_frame(C.byref(self.f), t, _ptr(out, f32p), threads)
            return out.reshape(Z, Y, X)
        bad = C.c_uint32()
        st = self.o.lib.vo_decode_frame(C.byref(self.f), t, _ptr(out, f32p), threads, C.byref(bad))
        if st:
            raise RuntimeError(f"oracle status {st} at leaf {bad.value}")
        return out.reshape(Z, Y, X)

    def page_table(self):
        compact = np.zeros(self.f.leaf_count, np.uint32)
        n = self.o.lib.vo_build_page_table(C.byref(self.f), _ptr(compact, u32p))
        return compact, int(n)

    def cache(self, t, threads=0):
        compact, n = self.page_table()
        out = np.zeros(max(n, 1) * 512, np.float32)
        st = self.o.lib.vo_decode_cache(C.byref(self.f), t, _ptr(compact, u32p), _ptr(out, f32p), threads)
        if st:
            raise RuntimeError(f"oracle status {st}")
        return out[: n * 512].reshape(n, 512)

    def control_cache(self, t, compact):
        """The Studio's 576-slot control cache of frame t (vbt_cache.comp), [active, 576]."""
        n = int(np.count_nonzero(compact != 0xFFFFFFFF))
        out = np.zeros(max(n, 1) * 576, np.float32)
        c = np.ascontiguousarray(compact, np.uint32)
        self.o.lib.vo_control_cache(C.byref(self.f), t, _ptr(c, u32p), _ptr(out, f32p))
        return out[: n * 576].reshape(n, 576)

    def sample_rays(self, cache, compact, params, rays):
        """The Studio's ray sampler (vbt_sample.comp): rays [n, 8] -> results [n, 8]."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        out = np.zeros_like(r)
        cc = np.ascontiguousarray(cache, np.float32).reshape(-1)
        c = np.ascontiguousarray(compact, np.uint32)
        self.o.lib.vo_sample_rays(C.byref(self.f), _ptr(cc, f32p), _ptr(c, u32p), C.byref(params), _ptr(r, f32p),
                                  r.shape[0], _ptr(out, f32p))
        return out

    def smoke_sample_rays(self, params, rays):
        """render/shaders/vbt_smoke_sample.comp over the payload: rays [n, 8] -> sums [n]."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        out = np.zeros(r.shape[0], np.float32)
        self.o.lib.vo_smoke_sample_rays(C.byref(self.f), C.byref(params), _ptr(r, f32p), r.shape[0], _ptr(out, f32p))
        return out

    def query(self, xyzt, threads=0):
        q = np.ascontiguousarray(xyzt, np.uint32)
        out = np.zeros(q.shape[0], np.float32)
        if self.profile == 2:
            self.o.lib.vo_sci_query_points(C.byref(self.f), _ptr(q, u32p), q.shape[0], _ptr(out, f32p), threads)
        else:
            st = self.o.lib.vo_query_points(C.byref(self.f), _ptr(q, u32p), q.shape[0], _ptr(out, f32p), threads)
            if st:
                raise RuntimeError(f"oracle status {st}")
        return out


class Reference:
    """The reference decoder compiled from its sources (oracle/_ref/libvbtref.so)."""

    def __init__(self):
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        L = self.lib = C.CDLL(REF_SO)
        L.vr_last_error.restype = C.c_char_p
        L.vr_load.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t]
        L.vr_load.restype = C.c_void_p
        L.vr_free.argtypes = [C.c_void_p]
        L.vr_decode_frame.argtypes = [C.c_void_p, C.c_int, f32p, C.c_int]
        L.vr_sci_frame.argtypes = [C.c_void_p, C.c_uint32, f32p]
        L.vr_sci_query.argtypes = [C.c_void_p, u32p, C.c_uint64, f32p, C.c_int]
        L.vr_decode_control.argtypes = [u8p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                                        C.c_int, C.c_uint32, C.c_int, f32p]
        L.vr_parse_leaf.argtypes = [u8p, C.c_size_t, u32p]
        L.vr_shell_voxel.argtypes = [u8p, C.c_size_t, C.c_int, C.c_uint32, C.c_int, f32p]
        L.vr_decode_leaf.argtypes = [u8p, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, f32p]
        L.vr_float_to_half.argtypes = [C.c_float]
        L.vr_float_to_half.restype = C.c_uint16
        L.vr_half_to_float.argtypes = [C.c_uint16]
        L.vr_half_to_float.restype = C.c_float
        L.vr_pack_stream.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, u32p, u8p, u32p, f32p,
                                     C.c_uint32, C.c_int, u8p, C.c_size_t]
        L.vr_pack_stream.restype = C.c_long
        L.vr_build_leaf.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u8p, C.c_size_t, u8p, C.c_size_t, u8p,
                                    C.c_size_t, C.c_int, u8p, C.c_size_t]
        L.vr_build_leaf.restype = C.c_long
        L.vr_pack_leaves.argtypes = [u8p, C.c_uint32, u32p, u8p, C.POINTER(C.c_uint16), f32p, u8p, u32p, u32p,
                                     C.c_size_t, C.c_int]
        L.vr_pack_leaves.restype = C.c_long
        L.vr_generate_queries.argtypes = [C.c_uint32] * 4 + [C.c_int, C.c_uint32, C.c_uint32, u32p, u32p]
        L.vr_dct.argtypes = [f32p, f32p, C.c_int, C.c_int, f32p, f32p]

    def generate_queries(self, dims, pattern, count, seed):
        """(generated, sorted) as [count, 5] arrays of (x, y, z, t, leafIndex)."""
        out = np.zeros((count, 5), np.uint32)
        srt = np.zeros((count, 5), np.uint32)
        self.lib.vr_generate_queries(*dims, pattern, count, seed, _ptr(out, u32p), _ptr(srt, u32p))
        return out, srt

    def dct(self, series, keep, weights=None):
        """(coeffs, decoded) of dctEncodeKeep[Weighted] and dctDecodeAt."""
        s = np.ascontiguousarray(series, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        coeffs = np.zeros(max(1, s.size), np.float32)
        dec = np.zeros(s.size, np.float32)
        k = self.lib.vr_dct(_ptr(s, f32p), None if w is None else _ptr(w, f32p), s.size, keep, _ptr(coeffs, f32p),
                            _ptr(dec, f32p))
        return coeffs[:k], dec

    def error(self):
        return self.lib.vr_last_error().decode()

    def load(self, path):
        err = C.create_string_buffer(512)
        h = self.lib.vr_load(path.encode(), err, 512)
        if not h:
            raise RuntimeError(err.value.decode())
        return h

    def free(self, h):
        self.lib.vr_free(h)

    def frame(self, h, dims, t, profile=1, threads=0):
        X, Y, Z = dims
        out = np.zeros(Z * Y * X, np.float32)
        if profile == 2:
            st = self.lib.vr_sci_frame(h, t, _ptr(out, f32p))
        else:
            st = self.lib.vr_decode_frame(h, t, _ptr(out, f32p), threads)
        if st:
            raise RuntimeError(self.error())
        return out.reshape(Z, Y, X)

    def sci_query(self, h, xyzt, threads=0):
        q = np.ascontiguousarray(xyzt, np.uint32)
        out = np.zeros(q.shape[0], np.float32)
        self.lib.vr_sci_query(h, _ptr(q, u32p), q.shape[0], _ptr(out, f32p), threads)
        return out

    def decode_control(self, stream, codec, cc, bins, kf, stream_bytes, total, ci, frame, align=True):
        s = np.ascontiguousarray(stream, np.uint8)
        out = C.c_float()
        st = self.lib.vr_decode_control(_ptr(s, u8p), codec, cc, bins, kf, stream_bytes, int(align), total, ci,
                                        frame, C.byref(out))
        return (self.error() if st else None), out.value

    def parse_leaf(self, leaf):
        b = np.ascontiguousarray(leaf, np.uint8)
        out = np.zeros(16, np.uint32)
        st = self.lib.vr_parse_leaf(_ptr(b, u8p), b.size, _ptr(out, u32p))
        return (self.error() if st else None), out

    def shell_voxel(self, leaf, total, voxel, frame):
        b = np.ascontiguousarray(leaf, np.uint8)
        out = C.c_float()
        st = self.lib.vr_shell_voxel(_ptr(b, u8p), b.size, total, voxel, frame, C.byref(out))
        return (self.error() if st else None), out.value

    def decode_leaf(self, leaf, total, frame, w=8, h=8, d=8):
        b = np.ascontiguousarray(leaf, np.uint8)
        out = np.zeros(w * h * d, np.float32)
        st = self.lib.vr_decode_leaf(_ptr(b, u8p), b.size, total, frame, w, h, d, _ptr(out, f32p))
        return (self.error() if st else None), out

    def pack_stream(self, codec, desc, bin_index, key_frames, key_values, bins, max_local=255, align=True):
        desc = np.ascontiguousarray(desc, np.uint32).reshape(-1)
        cc = desc.size // 3
        bi = np.ascontiguousarray(bin_index, np.uint8)
        kfr = np.ascontiguousarray(key_frames, np.uint32)
        kv = np.ascontiguousarray(key_values, np.float32)
        cap = 64 + cc * (4 + bins + 4) + kfr.size * 8 + 16
        out = np.zeros(cap, np.uint8)
        n = self.lib.vr_pack_stream(codec, cc, bins, max_local, _ptr(desc, u32p), _ptr(bi, u8p), _ptr(kfr, u32p),
                                    _ptr(kv, f32p), kfr.size, int(align), _ptr(out, u8p), cap)
        if n < 0:
            raise RuntimeError(self.error())
        return out[:n].copy()

    def pack_leaves(self, leaves, arr, threads=0):
        """(offsets, payload) of the reference's packer over the stream arrays of vbt_pack_leaves
        (leaves: 32-byte records as tests/leafstreams.py builds them)."""
        rec = np.ascontiguousarray(leaves).view(np.uint8)
        n = rec.size // 32
        desc = np.ascontiguousarray(arr["descriptors"], np.uint32)
        bins = np.ascontiguousarray(arr["bins"], np.uint8)
        kf = np.ascontiguousarray(arr["key_frames"], np.uint16)
        kv = np.ascontiguousarray(arr["key_values"], np.float32)
        occ = np.ascontiguousarray(arr["occupancy"], np.uint8)
        cap = 16 + 28 * n + desc.size + bins.size // 4 + 2 * kf.size
        off = np.zeros(n + 1, np.uint32)
        pay = np.zeros(cap, np.uint32)
        w = self.lib.vr_pack_leaves(_ptr(rec, u8p), n, _ptr(desc, u32p), _ptr(bins, u8p),
                                    _ptr(kf, C.POINTER(C.c_uint16)), _ptr(kv, f32p), _ptr(occ, u8p), _ptr(off, u32p),
                                    _ptr(pay, u32p), cap, threads)
        if w < 0:
            raise RuntimeError(self.error())
        return off, pay[:w]

    def build_leaf(self, packed_header, coarse_kf, fine_kf, coarse, fine, occ=None, align=True):
        c = np.ascontiguousarray(coarse, np.uint8)
        f = np.ascontiguousarray(fine, np.uint8)
        o = None if occ is None else np.ascontiguousarray(occ, np.uint8)
        cap = c.size + f.size + (0 if o is None else o.size) + 64
        out = np.zeros(cap, np.uint8)
        n = self.lib.vr_build_leaf(packed_header, coarse_kf, fine_kf, _ptr(c, u8p), c.size, _ptr(f, u8p), f.size,
                                   None if o is None else _ptr(o, u8p), 0 if o is None else o.size, int(align),
                                   _ptr(out, u8p), cap)
        if n < 0:
            raise RuntimeError(self.error())
        return out[:n].copy()


def _coarse_fit(fn, leaf_recon, extent, profile):
    lt = np.ascontiguousarray(leaf_recon, np.float32).reshape(512, -1)
    T = lt.shape[1]
    cap = 64 * max(T, 1)
    desc = np.zeros(64, np.uint32)
    bins = np.zeros((64, 8), np.uint8)
    kf = np.zeros(cap, np.uint16)
    kv = np.zeros(cap, np.float32)
    grid = np.zeros((64, T), np.float32)
    req = C.c_int()
    n = fn(_ptr(lt, f32p), T, *extent, C.byref(profile), _ptr(desc, u32p), _ptr(bins, u8p),
           _ptr(kf, C.POINTER(C.c_uint16)), _ptr(kv, f32p), cap, C.byref(req), _ptr(grid, f32p))
    if n < 0:
        raise RuntimeError("coarse fit: key capacity exceeded")
    return dict(desc=desc, bins=bins, key_frames=kf[:n].copy(), key_values=kv[:n].copy(),
                required_max_local=req.value, grid=grid)


class KeyframeReference:
    """The reference encoder's detectDensityKeyFrames / reconstructFromKeys, compiled from its source
    (oracle/_ref/libkfref.so, see kf_ref_shim.cpp)."""

    def __init__(self):
        if not os.path.exists(KFREF_SO):
            raise FileNotFoundError(KFREF_SO)
        L = self.lib = C.CDLL(KFREF_SO)
        i32p = C.POINTER(C.c_int)
        L.vbtref_detect_keyframes.argtypes = [f32p, C.c_int, C.POINTER(VoKeyframeProfile), i32p, i32p]
        L.vbtref_reconstruct.argtypes = [f32p, C.c_int, i32p, C.c_int, f32p]
        L.vbtref_coarse_fit.argtypes = [f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(VoKeyframeProfile), u32p,
                                        u8p, C.POINTER(C.c_uint16), f32p, C.c_int, C.POINTER(C.c_int), f32p]
        L.vbtref_temporal_pass.argtypes = [f32p, C.c_uint64, C.c_int, C.c_uint64, C.POINTER(VoKeyframeProfile),
                                           u32p, C.POINTER(C.c_double), C.c_int]

    def detect_keyframes(self, series, profile):
        v = np.ascontiguousarray(series, np.float32)
        keys = np.zeros(max(1, 4 * v.size + 4), np.int32)
        used = C.c_int()
        k = self.lib.vbtref_detect_keyframes(_ptr(v, f32p), v.size, C.byref(profile),
                                             _ptr(keys, C.POINTER(C.c_int)), C.byref(used))
        return keys[:k].copy(), bool(used.value)

    def reconstruct(self, series, keys):
        v = np.ascontiguousarray(series, np.float32)
        k = np.ascontiguousarray(keys, np.int32)
        out = np.zeros(v.size, np.float32)
        self.lib.vbtref_reconstruct(_ptr(v, f32p), v.size, _ptr(k, C.POINTER(C.c_int)), k.size, _ptr(out, f32p))
        return out

    def coarse_fit(self, leaf_recon, extent, profile):
        """The reference's coarse control fitting of one leaf (see Oracle.coarse_fit)."""
        return _coarse_fit(self.lib.vbtref_coarse_fit, leaf_recon, extent, profile)

    def temporal_pass(self, frames, profile, threads=0, series=None):
        """(key_count [S], err2 [S]) of the encoder's per-voxel loop over frames[T, S] (frame-major);
        `series` limits the pass to the first columns."""
        v = np.ascontiguousarray(frames, np.float32)
        T, S = v.shape
        n = S if series is None else int(series)
        kc = np.zeros(n, np.uint32)
        e2 = np.zeros(n, np.float64)
        self.lib.vbtref_temporal_pass(_ptr(v, f32p), n, T, S, C.byref(profile), _ptr(kc, u32p),
                                      _ptr(e2, C.POINTER(C.c_double)), threads)
        return kc, e2
