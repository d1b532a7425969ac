"""Control streams of a VBTPACK4 file's leaves, unpacked into the arrays vbt_pack_leaves reads
(test helper).

The leaves are parsed with computeRenderTemporalLeafLayout's arithmetic (restated below; the oracle's
parser checks it when given); each stream's
descriptors, bin index and keyframes are copied out as the encoder held them before
packRenderTemporalControlStream: descriptor words, 8 bin bytes per control (the first 4 for the
Mode2 residual stream's 4 bins), keyframe frames and values (FP16 values widened to float32).  A
stream's maxBinLocalKeys is not stored in the file; the smallest value its descriptors satisfy is
used (it only enters the packer's validation).
"""
import numpy as np

LEAF_DTYPE = np.dtype([("header", "<u4"), ("coarse_kf", "<u2"), ("fine_kf", "<u2"), ("coarse_control", "<u4"),
                       ("coarse_key", "<u4"), ("fine_control", "<u4"), ("fine_key", "<u4"), ("occupancy", "<u4"),
                       ("coarse_max_local", "u1"), ("fine_max_local", "u1"), ("pad", "u1", (2,))])
assert LEAF_DTYPE.itemsize == 32


def _align4(n):
    return (n + 3) & ~3


class _Builder:
    def __init__(self):
        self.desc, self.bins, self.frames, self.values, self.occ = [], [], [], [], []
        self.n_controls = self.n_keys = 0

    def stream(self, leaf, desc_off, controls, bins, key_off, keys, codec):
        d = np.frombuffer(leaf[desc_off:desc_off + 4 * controls].tobytes(), "<u4").copy()
        b = np.zeros((controls, 8), np.uint8)
        raw = leaf[desc_off + 4 * controls:desc_off + 4 * controls + controls * bins]
        b[:, :bins] = np.asarray(raw, np.uint8).reshape(controls, bins)
        if codec == 1:
            k = np.asarray(leaf[key_off:key_off + 8 * keys], np.uint8).reshape(keys, 8)
            fr = k[:, 0].astype(np.uint16) | (k[:, 1].astype(np.uint16) << 8)
            val = k[:, 4:8].copy().view("<f4").reshape(keys)
        else:
            k = np.asarray(leaf[key_off:key_off + 3 * keys], np.uint8).reshape(keys, 3)
            fr = k[:, 0].astype(np.uint16)
            hb = k[:, 1].astype(np.uint16) | (k[:, 2].astype(np.uint16) << 8)
            val = hb.view(np.float16).astype(np.float32)
        first_c, first_k = self.n_controls, self.n_keys
        self.desc.append(d)
        self.bins.append(b)
        self.frames.append(fr)
        self.values.append(val)
        self.n_controls += controls
        self.n_keys += keys
        count = (d >> 16) & 0xFF
        reserved = d >> 24
        max_local = max(1, int(reserved.max(initial=0)), int(-(-int(count.max(initial=0)) // bins)))
        return first_c, first_k, min(max_local, 255)

    def arrays(self):
        cat = lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(0, dt)  # noqa: E731
        return dict(descriptors=cat(self.desc, np.uint32),
                    bins=np.concatenate(self.bins).reshape(-1) if self.bins else np.zeros(0, np.uint8),
                    key_frames=cat(self.frames, np.uint16), key_values=cat(self.values, np.float32),
                    occupancy=np.concatenate(self.occ) if self.occ else np.zeros(0, np.uint8))


def _layout(leaf, word):
    """Offsets of a non-EMPTY leaf's sections (render_temporal_payload.cpp:143-197, and the Mode2
    residual stream after the occupancy, :348-386): (coarse_kf, fine_kf, coarse key offset,
    fine descriptor offset, fine key offset, active shell voxels)."""
    ckf, fkf = (int(x) for x in np.frombuffer(leaf[4:8].tobytes(), "<u2"))
    cres, fres = (word >> 6) & 7, (word >> 9) & 7
    stride = lambda codec: 8 if codec == 1 else 3  # noqa: E731
    cc = cres ** 3
    ckey = 8 + 4 * cc + _align4(8 * cc)
    fine = ckey + _align4(ckf * stride((word >> 2) & 3))
    mode = word & 3
    if mode == 3:
        fc = fres ** 3
        return ckf, fkf, ckey, fine, fine + 4 * fc + _align4(8 * fc), 0
    if mode == 2:
        act = int(np.unpackbits(np.asarray(leaf[fine:fine + 64], np.uint8)).sum())
        r0 = fine + 80
        return ckf, fkf, ckey, r0, r0 + 4 * act + _align4(4 * act), act
    return ckf, fkf, ckey, 0, 0, 0


def streams_from_file(path, oracle=None):
    """(leaves [L] LEAF_DTYPE, arrays dict, leaf byte blocks) of every leaf of the file.  With an
    oracle, every leaf's layout is checked against its parser."""
    raw = open(path, "rb").read()
    h = np.frombuffer(raw[8:52], np.uint32)
    leaf_count, scale_count = int(h[8]), int(h[10])
    off_at = 52 + 4 * scale_count
    offsets = np.frombuffer(raw[off_at:off_at + 4 * (leaf_count + 1)], np.uint32)
    pay_at = off_at + 4 * (leaf_count + 1)
    payload = np.frombuffer(raw, np.uint8, offset=pay_at)
    leaves = np.zeros(leaf_count, LEAF_DTYPE)
    b = _Builder()
    blocks = []
    for i in range(leaf_count):
        leaf = payload[4 * int(offsets[i]):4 * int(offsets[i + 1])]
        blocks.append(leaf.tobytes())
        word = int(np.frombuffer(leaf[:4].tobytes(), "<u4")[0])
        leaves[i]["header"] = word
        mode = word & 3
        if mode == 0:
            continue
        ckf, fkf, ckey, fdesc, fkey, act = _layout(leaf, word)
        if oracle is not None:
            st, v = oracle.parse_leaf(leaf)
            assert st == 0 and (v.coarse_kf, v.fine_kf, v.coarse.key_off) == (ckf, fkf, ckey), (path, i)
            if mode == 3:
                assert (v.fine.desc_off, v.fine.key_off) == (fdesc, fkey), (path, i)
            if mode == 2:
                assert (v.shell_residual_off, v.shell_active) == (fdesc, act), (path, i)
        cres, fres = (word >> 6) & 7, (word >> 9) & 7
        ccodec, fcodec = (word >> 2) & 3, (word >> 4) & 3
        leaves[i]["coarse_kf"], leaves[i]["fine_kf"] = ckf, fkf
        c = b.stream(leaf, 8, cres ** 3, 8, ckey, ckf, ccodec)
        leaves[i]["coarse_control"], leaves[i]["coarse_key"], leaves[i]["coarse_max_local"] = c
        if mode == 3:
            f = b.stream(leaf, fdesc, fres ** 3, 8, fkey, fkf, fcodec)
            leaves[i]["fine_control"], leaves[i]["fine_key"], leaves[i]["fine_max_local"] = f
        elif mode == 2:
            leaves[i]["occupancy"] = len(b.occ)
            b.occ.append(np.asarray(leaf[fdesc - 80:fdesc], np.uint8).copy())
            f = b.stream(leaf, fdesc, act, 4, fkey, fkf, fcodec)
            leaves[i]["fine_control"], leaves[i]["fine_key"], leaves[i]["fine_max_local"] = f
    return leaves, b.arrays(), blocks
