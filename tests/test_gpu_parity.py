"""GPU parity: the sm_100a kernels (through the C-ABI) against the oracle and the golden fixtures.

Render-temporal outputs (leaf table, page table, frames, caches, point and slice queries) must be
bit-exact.  Scientific outputs must be within 1e-6 of the field range (the reference sums the
coarse DCT in double; the GPU uses compensated float-float sums), and the test also reports how
many values are bit-exact.
"""
import os

import numpy as np
import pytest

from conftest import ASSETS, GOLDEN, golden_asset

pytestmark = pytest.mark.gpu

SCI_TOL = 1e-6   # relative to the field range


GOLDEN_NAMES = ("tiny_density", "tiny_levelset", "sci_small", "sci_coarse", "sci_dense", "sci_dense_tb")


def asset_paths(include_large=False):
    out = [golden_asset(n) for n in GOLDEN_NAMES]
    names = ["cfg1_blobs", "cfg4_sdf_small", "sci_64", "sci_modes"] + (["cfg2_plume"] if include_large else [])
    for n in names:
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


def same_bits(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


def check_values(profile, got, want, rng_scale, what):
    if profile == 2:
        err = np.abs(got.astype(np.float64) - want.astype(np.float64))
        assert err.max(initial=0.0) <= SCI_TOL * rng_scale, (what, float(err.max()), rng_scale)
    else:
        bad = np.flatnonzero(got.reshape(-1).view(np.uint32) != want.reshape(-1).view(np.uint32))
        assert bad.size == 0, (what, bad[:8], got.reshape(-1)[bad[:8]], want.reshape(-1)[bad[:8]])


@pytest.fixture(scope="module")
def loaded(vbt, cuda, oracle):
    cache = {}

    def get(path):
        if path not in cache:
            a = vbt.Asset(path)
            f = oracle.load(path)
            cache[path] = (a, f)
        return cache[path]

    yield get
    for a, _ in cache.values():
        a.close()


def field_range(f):
    lo, hi = np.inf, -np.inf
    for t in range(0, f.frames, max(1, f.frames // 8)):
        fr = f.frame(t, threads=8)
        lo, hi = min(lo, float(fr.min())), max(hi, float(fr.max()))
    return max(hi - lo, 1e-30)


@pytest.mark.parametrize("path", asset_paths(True), ids=os.path.basename)
def test_page_table_and_leaf_table(loaded, path):
    a, f = loaded(path)
    compact, n = a.page_table()
    want, wn = f.page_table()
    assert n == wn and np.array_equal(compact, want)
    rows = a.leaf_table()
    off, pay = f.offsets(), f.payload()
    assert np.array_equal(rows[:, 0], off[:-1])
    assert np.array_equal(rows[:, 1] & 3, pay[off[:-1]] & 3) or f.profile == 2
    if f.profile != 2:
        assert np.array_equal(rows[:, 1], pay[off[:-1]])
        # every leaf parses as the oracle parses it: counts, layout, Mode2 active count, status
        raw = pay.view(np.uint8)
        for leaf in range(0, f.leaf_count, max(1, f.leaf_count // 2048)):
            b0, b1 = 4 * int(off[leaf]), 4 * int(off[leaf + 1])
            st, v = f.o.parse_leaf(raw[b0:b1])
            assert (rows[leaf, 7] >> 16) & 0xFF == st
            if st == 0 and v.header.mode != 0:
                assert rows[leaf, 2] == v.coarse_kf | (v.fine_kf << 16)
                assert rows[leaf, 3] == v.coarse.total
                if v.header.mode == 2:
                    assert rows[leaf, 7] & 0x3FF == v.shell_active
                    assert rows[leaf, 5] == v.shell_residual_off and rows[leaf, 6] == v.shell_residual_bytes


@pytest.mark.parametrize("path", asset_paths(), ids=os.path.basename)
def test_dense_frames(loaded, cuda, path):
    a, f = loaded(path)
    X, Y, Z = f.dims
    ts = list(range(f.frames)) if f.profile == 2 else list(range(-1, f.frames + 1))
    scale = field_range(f) if f.profile == 2 else 1.0
    out = cuda.empty((len(ts), Z, Y, X), dtype=cuda.float32, device="cuda")
    for i in range(0, len(ts), 16):
        chunk = ts[i:i + 16]
        a.decode_frames(chunk, out[i:i + len(chunk)])
    a.sync_status()
    got = out.cpu().numpy()
    exact = 0
    for i, t in enumerate(ts):
        want = f.frame(t, threads=8)
        check_values(f.profile, got[i], want, scale, (os.path.basename(path), t))
        exact += int(same_bits(got[i], want))
    if f.profile != 2:
        assert exact == len(ts)


def test_golden_frames_against_reference_fixtures(vbt, cuda):
    """The reference's own frames (tests/golden/assets/*.npz), independent of the oracle: every
    render leaf route and every scientific leaf mode (CoarseOnly, SparseEvents, DenseGrid3/4 with
    the per-frame BFP and the temporal-basis residual)."""
    for name in GOLDEN_NAMES:
        a = vbt.Asset(golden_asset(name))
        z = np.load(os.path.join(GOLDEN, "assets", name + ".npz"))
        X, Y, Z = a.dims
        ts = [int(t) for t in z["t"]]
        out = cuda.empty((len(ts), Z, Y, X), dtype=cuda.float32, device="cuda")
        a.decode_frames(ts, out)
        a.sync_status()
        got = out.cpu().numpy()
        want = z["frames"]
        if a.profile == 2:
            rng_scale = float(want.max() - want.min())
            assert np.abs(got.astype(np.float64) - want).max() <= SCI_TOL * rng_scale
        else:
            assert same_bits(got, want), name
        a.close()


@pytest.mark.parametrize("path", asset_paths(True), ids=os.path.basename)
def test_cache_batched_and_plain(loaded, cuda, path):
    a, f = loaded(path)
    n = a.active_count
    frames = [0, f.frames // 2, f.frames - 1] if f.profile == 2 else [-3, 0, f.frames // 3, f.frames - 1, f.frames + 4]
    cache = cuda.empty((len(frames), max(n, 1), 512), dtype=cuda.float32, device="cuda")
    a.build_page_table()
    a.decode_cache(frames, cache)
    plain = cuda.empty((max(n, 1), 512), dtype=cuda.float32, device="cuda")
    a.decode_cache_plain(frames[1], plain)
    a.sync_status()
    got = cache.cpu().numpy()[:, :n]
    scale = field_range(f) if f.profile == 2 else 1.0
    for i, t in enumerate(frames):
        want = f.cache(t, threads=8)
        check_values(f.profile, got[i], want, scale, (os.path.basename(path), t))
    assert same_bits(plain.cpu().numpy()[:n], got[1])


@pytest.mark.parametrize("path", asset_paths(), ids=os.path.basename)
def test_point_queries(loaded, cuda, path):
    a, f = loaded(path)
    rng = np.random.default_rng(11)
    nq = 100_000 if "cfg1" in path else 20_000
    X, Y, Z = f.dims
    tmax = f.frames if f.profile == 2 else f.frames + 3
    tmin = 0 if f.profile == 2 else -2
    q = np.stack([rng.integers(0, X, nq), rng.integers(0, Y, nq), rng.integers(0, Z, nq),
                  rng.integers(tmin, tmax, nq)], 1).astype(np.int64).astype(np.uint32)
    dq = cuda.from_numpy(q.view(np.int32)).cuda()
    out = cuda.empty(nq, dtype=cuda.float32, device="cuda")
    a.query_points(dq, out)
    a.sync_status()
    want = f.query(q.astype(np.int32).astype(np.uint32) if f.profile == 2 else q, threads=8)
    scale = field_range(f) if f.profile == 2 else 1.0
    check_values(f.profile, out.cpu().numpy(), want, scale, os.path.basename(path))
    # the host-buffer call returns the same values
    host_out = np.zeros(nq, np.float32)
    a.query_points_host(np.ascontiguousarray(q), host_out)
    assert same_bits(host_out, out.cpu().numpy())


@pytest.mark.parametrize("path", asset_paths(), ids=os.path.basename)
def test_slice_queries(loaded, cuda, path):
    a, f = loaded(path)
    X, Y, Z = f.dims
    t0, t1 = (0, f.frames) if f.profile == 2 else (-1, f.frames + 1)
    scale = field_range(f) if f.profile == 2 else 1.0
    for z in sorted({0, Z // 2, Z - 1}):
        out = cuda.zeros((t1 - t0, Y, X), dtype=cuda.float32, device="cuda")
        a.query_slice(z, t0, t1, out)
        a.sync_status()
        got = out.cpu().numpy()
        for i, t in enumerate(range(t0, t1)):
            check_values(f.profile, got[i], f.frame(t, threads=8)[z], scale, (os.path.basename(path), z, t))


def test_mode2_signs_bit_exact(loaded, cuda):
    """phi = 0 sign checks on the level-set assets: every voxel's sign (and value) as the oracle."""
    paths = [golden_asset("tiny_levelset")] + [p for p in asset_paths() if "cfg4" in p]
    for path in paths:
        a, f = loaded(path)
        X, Y, Z = f.dims
        out = cuda.empty((f.frames, Z, Y, X), dtype=cuda.float32, device="cuda")
        for i in range(0, f.frames, 16):
            ts = list(range(i, min(f.frames, i + 16)))
            a.decode_frames(ts, out[i:i + len(ts)])
        a.sync_status()
        got = out.cpu().numpy()
        for t in range(f.frames):
            want = f.frame(t, threads=8)
            assert np.array_equal(np.signbit(got[t]), np.signbit(want))
            assert np.array_equal(got[t] > 0, want > 0)


def test_control_values_golden_streams(vbt, cuda):
    """The checked scalar decode on the reference tests' streams (both codecs, 4/8 bins, corrupted
    hints, t = -2..T+2) equals the reference's values bit for bit."""
    z = np.load(os.path.join(GOLDEN, "streams.npz"))
    meta, blob, ts, ref = z["meta"], z["bytes"], z["t"], z["ref"]
    pos = 0
    for codec, bins, frames, kf, nbytes, off, nt in meta:
        stream = cuda.from_numpy(np.ascontiguousarray(blob[off:off + nbytes])).cuda()
        t = cuda.from_numpy(ts[pos:pos + nt].astype(np.int32)).cuda()
        ci = cuda.zeros(int(nt), dtype=cuda.int32, device="cuda")
        out = cuda.empty(int(nt), dtype=cuda.float32, device="cuda")
        st = cuda.empty(int(nt), dtype=cuda.int32, device="cuda")
        vbt.decode_control_values(stream, int(nbytes), int(codec), 1, int(bins), int(kf), int(frames), ci, t,
                                  int(nt), out, st)
        cuda.cuda.synchronize()
        assert int(st.abs().max()) == 0
        assert same_bits(out.cpu().numpy(), ref[pos:pos + nt]), (codec, bins, frames)
        pos += nt


def test_control_values_errors(vbt, cuda, oracle):
    """Error statuses of the checked scalar decode equal the oracle's on malformed calls."""
    z = np.load(os.path.join(GOLDEN, "streams.npz"))
    meta, blob = z["meta"], z["bytes"]
    codec, bins, frames, kf, nbytes, off, _ = (int(x) for x in meta[5])
    s = np.ascontiguousarray(blob[off:off + nbytes])
    cases = [(1, kf, nbytes, 0), (1, kf, nbytes - 4, 0), (1, kf + 400, nbytes, 0), (1, kf, nbytes, 3)]
    stream = cuda.from_numpy(s).cuda()
    for cc, kfc, nb, ci in cases:
        want_st, want_v = oracle.decode_control(s, codec, cc, bins, kfc, nb, frames, ci, 5)
        d_ci = cuda.tensor([ci], dtype=cuda.int32, device="cuda")
        d_t = cuda.tensor([5], dtype=cuda.int32, device="cuda")
        out = cuda.empty(1, dtype=cuda.float32, device="cuda")
        st = cuda.empty(1, dtype=cuda.int32, device="cuda")
        vbt.decode_control_values(stream, nb, codec, cc, bins, kfc, frames, d_ci, d_t, 1, out, st)
        cuda.cuda.synchronize()
        assert int(st.item()) == want_st, (cc, kfc, nb, ci)


def test_corrupted_asset_reports_leaf_status(vbt, cuda, oracle):
    """A corrupted Mode2 leaf: the walker records the parser's status for that leaf, decode calls
    report it through vbt_asset_sync_status, and every other leaf still decodes bit-exact."""
    path = golden_asset("tiny_levelset")
    raw = bytearray(open(path, "rb").read())
    f = oracle.load(path)
    off, pay = f.offsets(), f.payload()
    hdr_bytes = 52 + 4 * 0 + 4 * (f.leaf_count + 1)
    mode2 = [l for l in range(f.leaf_count) if (pay[off[l]] & 3) == 2]
    leaf = mode2[0]
    st, v = f.o.parse_leaf(pay.view(np.uint8)[4 * off[leaf]:4 * off[leaf + 1]])
    occ = hdr_bytes + 4 * int(off[leaf]) + v.fine.desc_off
    raw[occ + 64 + 2:occ + 64 + 4] = b"\xff\x7f"          # group prefix of group 1
    a = vbt.Asset(data=bytes(raw))
    rows = a.leaf_table()
    assert (rows[leaf, 7] >> 16) & 0xFF == 5               # "group prefix is inconsistent"
    X, Y, Z = a.dims
    out = cuda.empty((1, Z, Y, X), dtype=cuda.float32, device="cuda")
    a.decode_frames([3], out)
    with pytest.raises(vbt.VbtError) as ei:
        a.sync_status()
    assert ei.value.status == 5 and f"leaf {leaf}" in ei.value.message
    want = f.frame(3)
    got = out.cpu().numpy()[0]
    lcx, lcy = (X + 7) // 8, (Y + 7) // 8
    bz, by, bx = leaf // (lcx * lcy), (leaf // lcx) % lcy, leaf % lcx
    m = np.ones_like(want, bool)
    m[bz * 8:bz * 8 + 8, by * 8:by * 8 + 8, bx * 8:bx * 8 + 8] = False
    assert same_bits(got[m], want[m])
    a.sync_status()   # error was cleared
    a.close()


def test_unsorted_keys_and_descending_frames(vbt, cuda, oracle, tmp_path):
    """Leaves whose key frames are not strictly increasing (here: one key frame byte rewritten)
    lose the sorted flag and take the reference-search path; descending frame lists take it too.
    Both must stay bit-exact with the oracle."""
    path = golden_asset("tiny_density")
    raw = bytearray(open(path, "rb").read())
    f = oracle.load(path)
    off, pay = f.offsets(), f.payload()
    hdr_bytes = 52 + 4 * (f.leaf_count + 1)
    leaf = int(np.flatnonzero((pay[off[:-1]] & 3) != 0)[0])
    st, v = f.o.parse_leaf(pay.view(np.uint8)[4 * off[leaf]:4 * off[leaf + 1]])
    leaf0 = hdr_bytes + 4 * int(off[leaf])
    desc = np.frombuffer(bytes(raw[leaf0 + 8:leaf0 + 8 + 4 * 64]), np.uint32)
    c = int(np.flatnonzero(((desc >> 16) & 0xFF) >= 2)[0])
    ks = int(desc[c] & 0xFFFF)
    kb = leaf0 + v.coarse.key_off
    raw[kb + 3 * (ks + 1)] = raw[kb + 3 * ks]          # duplicate the first key's frame
    path2 = str(tmp_path / "unsorted_tiny.vbtp")
    open(path2, "wb").write(raw)
    a = vbt.Asset(data=bytes(raw))
    f2 = oracle.load(path2)
    rows = a.leaf_table()
    assert (rows[leaf, 7] & (1 << 14)) == 0                 # not flagged sorted
    others = (rows[:, 7] & (1 << 10)) != 0
    others[leaf] = False
    assert np.all((rows[others, 7] & (1 << 14)) != 0)      # every other active leaf is
    X, Y, Z = a.dims
    for ts in (list(range(-1, a.frames + 1)), list(range(a.frames, -2, -1))):
        out = cuda.empty((len(ts), Z, Y, X), dtype=cuda.float32, device="cuda")
        a.decode_frames(ts, out)
        a.sync_status()
        got = out.cpu().numpy()
        for i, t in enumerate(ts):
            assert same_bits(got[i], f2.frame(t)), t
    a.close()


def test_event_on_masked_out_voxel(vbt, cuda, oracle, tmp_path):
    """A SparseEvents leaf with an event on a voxel whose mask bit is clear: the reference's mask
    test hides that event, so the leaf loses the sorted flag (no scatter of its events) and the
    per-frame, cache and window decodes still agree with the oracle."""
    path = golden_asset("sci_small")
    raw = bytearray(open(path, "rb").read())
    f = oracle.load(path)
    off, pay = f.offsets(), f.payload()
    p0 = bytes(raw).find(pay.tobytes())
    hdr = pay[off[:-1]]
    leaf = int(np.flatnonzero(((hdr & 3) == 1) & (((hdr >> 16) & 0xFFF) > 0))[0])
    h = int(hdr[leaf])
    keep = ((h >> 2) & 0x3F) + 1
    sb = p0 + 4 * int(off[leaf]) + 4 + 64 * (keep + 1)
    bins = np.frombuffer(bytes(raw[sb + 68:sb + 100]), np.uint16)
    e0 = int(bins[int(np.flatnonzero(np.append(bins[1:], (h >> 16) & 0xFFF) > bins)[0])])
    key = int(np.frombuffer(bytes(raw[sb + 100 + 2 * e0:sb + 102 + 2 * e0]), np.uint16)[0])
    li = key & 511
    mw = sb + 4 + 4 * (li >> 5)
    word = int(np.frombuffer(bytes(raw[mw:mw + 4]), np.uint32)[0]) & ~(1 << (li & 31))
    raw[mw:mw + 4] = np.uint32(word).tobytes()
    path2 = str(tmp_path / "masked_event.vbtp")
    open(path2, "wb").write(raw)
    a = vbt.Asset(data=bytes(raw))
    f2 = oracle.load(path2)
    rows = a.leaf_table()
    assert (rows[leaf, 7] & (1 << 14)) == 0
    X, Y, Z = a.dims
    ts = list(range(a.frames))
    out = cuda.empty((len(ts), Z, Y, X), dtype=cuda.float32, device="cuda")
    a.decode_frames(ts, out)
    a.sync_status()
    got = out.cpu().numpy()
    for i, t in enumerate(ts):
        assert same_bits(got[i], f2.frame(t)), t
    L = a.leaf_count
    exact = cuda.empty((len(ts), L, 512), dtype=cuda.float32, device="cuda")
    a.decode_cache(ts, exact, frame_stride=L * 512)
    win = cuda.empty((len(ts), L, 512), dtype=cuda.float32, device="cuda")
    a.decode_window(0, len(ts), win)
    a.sync_status()
    e, w = exact.cpu().numpy(), win.cpu().numpy()
    mx, _, lo, hi = a.window_error(0, len(ts), win)
    assert np.abs(w.astype(np.float64) - e).max() <= 1e-6 * (hi - lo)
    assert mx <= 1e-6 * (hi - lo)
    a.close()


@pytest.mark.parametrize("name", ["cfg2_plume", "mix_fire_flames"])
def test_point_queries_sparse_volume(oracle, cuda, vbt, name):
    """Volumes whose leaves are mostly EMPTY take the compacting point-query kernel (trivial
    queries answered first, the rest decoded from a per-CTA list); values equal the oracle's, also
    through the merged serving launch."""
    p = os.path.join(ASSETS, name + ".vbtp")
    if not os.path.exists(p):
        pytest.skip(f"{name} not generated")
    f = oracle.load(p)
    a = vbt.Asset(p)
    rng = np.random.default_rng(17)
    X, Y, Z = a.dims
    for nq in (1000, 300_000):
        q = np.stack([rng.integers(0, X, nq), rng.integers(0, Y, nq), rng.integers(0, Z, nq),
                      rng.integers(-2, a.frames + 2, nq)], 1).astype(np.int64).astype(np.uint32)
        dq = cuda.from_numpy(q.view(np.int32)).cuda()
        out = cuda.empty(nq, dtype=cuda.float32, device="cuda")
        a.query_points(dq, out)
        a.sync_status()
        got = out.cpu().numpy()
        want = f.query(q, threads=8)
        assert same_bits(got, want), name
        srv = vbt.Server(hbm_budget_bytes=256 << 20, slots=2)
        sid = srv.add_asset(a)
        ho = np.zeros(nq, np.float32)
        t = srv.submit_points(sid, np.ascontiguousarray(q), ho)
        assert srv.wait(t).status == 0
        srv.release(t)
        srv.close()
        assert same_bits(ho, want), name
    a.close()


@pytest.mark.parametrize("path", [p for p in asset_paths() if "sci" not in os.path.basename(p)],
                         ids=os.path.basename)
def test_control_cache(loaded, oracle, cuda, path):
    """The Studio's 576-slot control cache: every slot of sampled active leaves equals the oracle's
    control decode (coarse in slots 0..63, fine or Mode2 shell controls from 64, zeros elsewhere)."""
    a, f = loaded(path)
    a.build_page_table()
    compact, n = a.page_table()
    frames = [-1, 0, f.frames // 2, f.frames - 1, f.frames + 2]
    out = cuda.full((len(frames), max(n, 1), 576), float("nan"), dtype=cuda.float32, device="cuda")
    a.decode_control_cache(frames, out, frame_stride=max(n, 1) * 576)
    a.sync_status()
    got = out.cpu().numpy()
    off, pay = f.offsets(), f.payload()
    raw = pay.view(np.uint8)
    leaves = np.flatnonzero(compact != 0xFFFFFFFF)
    assert len(leaves) == n
    for leaf in leaves[::max(1, len(leaves) // 16)]:
        blk = raw[4 * int(off[leaf]):4 * int(off[leaf + 1])]
        st, v = oracle.parse_leaf(blk)
        assert st == 0
        h = v.header

        def ctrl(start, nbytes, codec, cc, bins, kf, ci, t):
            s, val = oracle.decode_control(blk[start:start + nbytes], codec, cc, bins, kf, nbytes, f.frames, ci, t)
            assert s == 0
            return val

        for j, t in enumerate(frames):
            want = np.zeros(576, np.float32)
            cc = h.coarse_res ** 3
            for s in range(min(64, cc)):
                want[s] = ctrl(v.coarse_off, v.coarse.total, h.coarse_codec, cc, 8, v.coarse_kf, s, t)
            if h.mode == 3:
                cf = h.fine_res ** 3
                for ci in range(min(512, cf)):
                    want[64 + ci] = ctrl(v.fine_off, v.fine.total, h.fine_codec, cf, 8, v.fine_kf, ci, t)
            elif h.mode == 2:
                for ci in range(min(512, v.shell_active)):
                    want[64 + ci] = ctrl(v.shell_residual_off, v.shell_residual_bytes, h.fine_codec,
                                         v.shell_active, 4, v.fine_kf, ci, t)
            assert same_bits(got[j, compact[leaf]], want), (os.path.basename(path), int(leaf), t)
