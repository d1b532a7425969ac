"""The serving loop (vbt_server_* / vbt_serve_*): every result is the same alone and in a mix,
admission respects the HBM budget, per-request statuses survive merging, device-resident results
stay valid until release.

Requests are point batches, z-slices over frame ranges and dense frames over several resident
assets (render-temporal, Mode2 level set, scientific).  "Alone" means a plain server (one request
per launch, one launch in flight); "mix" means all requests submitted at once from several
threads to a server with 4 streams that merges point requests across assets.  Results must be
bit-identical, and equal to the one-asset C-ABI calls and to the oracle.
"""
import ctypes as C
import os
import threading

import numpy as np
import pytest

from conftest import ASSETS, golden_asset

pytestmark = pytest.mark.gpu

NAMES = ["tiny_density", "tiny_levelset", "sci_small"]


def asset_paths():
    out = [golden_asset(n) for n in NAMES]
    for n in ("cfg1_blobs", "cfg4_sdf_small"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


@pytest.fixture(scope="module")
def assets(vbt, cuda):
    objs = [vbt.Asset(p) for p in asset_paths()]
    yield objs
    for a in objs:
        a.close()


def make_requests(assets, seed=3, n=60):
    """A seeded mix: 70% point batches, 20% slices, 10% dense frames."""
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n):
        i = int(rng.integers(len(assets)))
        a = assets[i]
        X, Y, Z = a.dims
        T = a.frames
        u = rng.random()
        if u < 0.7:
            m = int(rng.integers(1, 5000))
            q = np.stack([rng.integers(0, X, m), rng.integers(0, Y, m), rng.integers(0, Z, m),
                          rng.integers(0, T, m)], axis=1).astype(np.uint32)
            reqs.append(("points", i, np.ascontiguousarray(q)))
        elif u < 0.9:
            t0 = int(rng.integers(0, T))
            t1 = min(T, t0 + int(rng.integers(1, 6)))
            reqs.append(("slice", i, (int(rng.integers(0, Z)), t0, t1)))
        else:
            fr = [int(x) for x in rng.integers(0, T, int(rng.integers(1, 4)))]
            reqs.append(("frames", i, fr))
    return reqs


def out_size(a, req):
    kind, _, arg = req
    X, Y, Z = a.dims
    if kind == "points":
        return arg.shape[0]
    if kind == "slice":
        return (arg[2] - arg[1]) * X * Y
    return len(arg) * X * Y * Z


def submit(server, ids, req, out):
    kind, i, arg = req
    if kind == "points":
        return server.submit_points(ids[i], arg, out)
    if kind == "slice":
        return server.submit_slice(ids[i], arg[0], arg[1], arg[2], out)
    return server.submit_frames(ids[i], arg, out)


def pinned_empty(cuda, n):
    t = cuda.empty(max(n, 1), dtype=cuda.float32, pin_memory=True)
    return t, t.numpy()[:n]


def run_alone(vbt, cuda, assets, reqs):
    srv = vbt.Server(hbm_budget_bytes=256 << 20, plain=True)
    ids = [srv.add_asset(a) for a in assets]
    outs = []
    for r in reqs:
        keep, out = pinned_empty(cuda, out_size(assets[r[1]], r))
        t = submit(srv, ids, r, out)
        res = srv.wait(t)
        assert res.status == 0, (r[0], res.status)
        srv.release(t)
        outs.append(out.copy())
    srv.close()
    return outs


def test_alone_equals_mix_and_one_asset_calls(vbt, cuda, assets, oracle):
    reqs = make_requests(assets)
    alone = run_alone(vbt, cuda, assets, reqs)

    srv = vbt.Server(hbm_budget_bytes=256 << 20, slots=4)
    ids = [srv.add_asset(a) for a in assets]
    bufs = [pinned_empty(cuda, out_size(assets[r[1]], r)) for r in reqs]
    tickets = [None] * len(reqs)

    def client(k):
        for j in range(k, len(reqs), 4):
            tickets[j] = submit(srv, ids, reqs[j], bufs[j][1])

    th = [threading.Thread(target=client, args=(k,)) for k in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for j, t in enumerate(tickets):
        res = srv.wait(t)
        assert res.status == 0, (reqs[j][0], res.status)
        srv.release(t)
    st = srv.stats()
    assert st.requests_done == len(reqs)
    assert st.p99_ms >= st.p50_ms > 0.0
    srv.close()

    for j, r in enumerate(reqs):
        assert np.array_equal(bufs[j][1].view(np.uint32), alone[j].view(np.uint32)), (j, r[0])

    # the one-asset calls and the oracle give the same values
    for j, r in enumerate(reqs):
        kind, i, arg = r
        a = assets[i]
        X, Y, Z = a.dims
        if kind == "points":
            want = np.empty(arg.shape[0], np.float32)
            a.query_points_host(arg, want)
        elif kind == "slice":
            d = cuda.empty((arg[2] - arg[1]) * X * Y, dtype=cuda.float32, device="cuda")
            a.query_slice(arg[0], arg[1], arg[2], d)
            want = d.cpu().numpy()
        else:
            d = cuda.empty((len(arg), Z, Y, X), dtype=cuda.float32, device="cuda")
            a.decode_frames(arg, d)
            want = d.cpu().numpy().reshape(-1)
        a.sync_status()
        assert np.array_equal(bufs[j][1].view(np.uint32), want.view(np.uint32)), (j, kind)
        if kind == "points" and a.profile != 2:
            f = oracle.load(asset_paths()[i])
            assert np.array_equal(f.query(arg).view(np.uint32), want.view(np.uint32))


def test_point_requests_merge_into_one_launch(vbt, cuda, assets):
    """Point requests pending together on several assets go out as one launch."""
    srv = vbt.Server(hbm_budget_bytes=96 << 20, slots=1)
    ids = [srv.add_asset(a) for a in assets]
    big = assets[0]
    X, Y, Z = big.dims
    # a large point request (pageable input, staged by the scheduler) occupies the only stream
    # while the small requests queue up behind it
    n = 1 << 21
    r0 = np.random.default_rng(0)
    hq = np.stack([r0.integers(0, X, n), r0.integers(0, Y, n), r0.integers(0, Z, n),
                   r0.integers(0, big.frames, n)], axis=1).astype(np.uint32)
    hold = srv.submit_points(ids[0], hq, np.empty(n, np.float32))
    rng = np.random.default_rng(1)
    ts, outs = [], []
    for i, a in enumerate(assets):
        ax, ay, az = a.dims
        q = np.stack([rng.integers(0, ax, 300), rng.integers(0, ay, 300), rng.integers(0, az, 300),
                      rng.integers(0, a.frames, 300)], axis=1).astype(np.uint32)
        o = np.empty(300, np.float32)
        ts.append(srv.submit_points(ids[i], q, o))
        outs.append((a, q, o))
    srv.wait(hold)
    srv.release(hold)
    for t in ts:
        assert srv.wait(t).status == 0
        srv.release(t)
    st = srv.stats()
    assert st.units < 1 + len(assets), st.units   # the small requests shared a launch
    for a, q, o in outs:
        want = np.empty(q.shape[0], np.float32)
        a.query_points_host(q, want)
        a.sync_status()
        assert np.array_equal(o.view(np.uint32), want.view(np.uint32))
    srv.close()


def test_budget_admission_and_limit(vbt, cuda, assets):
    a = assets[0]
    X, Y, Z = a.dims
    frame_bytes = (4 * X * Y * Z + 255) // 256 * 256
    budget = 3 * (frame_bytes + 256)               # room for 3 single-frame units (result + error word)
    srv = vbt.Server(hbm_budget_bytes=budget, slots=8)
    aid = srv.add_asset(a)
    with pytest.raises(vbt.VbtError) as ei:
        srv.submit_frames(aid, list(range(4)), np.empty(4 * X * Y * Z, np.float32))
    assert ei.value.status == 43
    outs = [pinned_empty(cuda, X * Y * Z) for _ in range(24)]
    ts = [srv.submit_frames(aid, [k % a.frames], outs[k][1]) for k in range(24)]
    for t in ts:
        assert srv.wait(t).status == 0
        srv.release(t)
    st = srv.stats()
    assert st.arena_peak_bytes <= budget and st.requests_done == 24
    d = cuda.empty((1, Z, Y, X), dtype=cuda.float32, device="cuda")
    for k in range(24):
        a.decode_frames([k % a.frames], d)
        assert np.array_equal(outs[k][1].view(np.uint32), d.cpu().numpy().reshape(-1).view(np.uint32))
    srv.close()


def test_status_per_request(vbt, cuda, assets):
    """A scientific point request with t >= frames fails with DECODE_OOB; a render request
    submitted right after it (merged into the same launch when both are pending together) still
    succeeds."""
    sci = [a for a in assets if a.profile == 2][0]
    rt = [a for a in assets if a.profile != 2][0]
    srv = vbt.Server(hbm_budget_bytes=64 << 20, slots=1, max_batch_queries=1 << 20)
    i_sci, i_rt = srv.add_asset(sci), srv.add_asset(rt)
    bad = np.array([[1, 1, 1, sci.frames + 2]] * 8, np.uint32)
    good = np.array([[1, 2, 3, 0]] * 8, np.uint32)
    ob, og = np.empty(8, np.float32), np.empty(8, np.float32)
    tb = srv.submit_points(i_sci, bad, ob)
    tg = srv.submit_points(i_rt, good, og)
    rb, rg = srv.wait(tb), srv.wait(tg)
    assert rb.status == 11 and rg.status == 0
    srv.release(tb)
    srv.release(tg)
    srv.close()


def test_device_resident_results(vbt, cuda, assets):
    a = assets[0]
    X, Y, Z = a.dims
    srv = vbt.Server(hbm_budget_bytes=64 << 20, slots=2)
    aid = srv.add_asset(a)
    t = srv.submit_slice(aid, Z // 2, 0, 2)
    res = srv.wait(t)
    assert res.status == 0 and res.device_result and res.result_floats == 2 * X * Y
    path = "/usr/local/cuda/lib64/libcudart.so.12"
    if not os.path.exists(path):
        pytest.skip("libcudart not found for the device-to-host copy")
    cudart = C.CDLL(path)
    got = np.empty(res.result_floats, np.float32)
    assert cudart.cudaMemcpy(C.c_void_p(got.ctypes.data), C.c_void_p(res.device_result),
                             C.c_size_t(got.nbytes), 2) == 0
    d = cuda.empty(2 * X * Y, dtype=cuda.float32, device="cuda")
    a.query_slice(Z // 2, 0, 2, d)
    assert np.array_equal(got.view(np.uint32), d.cpu().numpy().view(np.uint32))
    srv.release(t)
    srv.close()


def test_device_resident_requests(vbt, cuda, assets):
    """A client that keeps its query batches and results on the GPU: point inputs in device memory,
    results written to device buffers (and slices/frames into device buffers), merged with host
    requests in one server; every result equals the host-buffer path bit for bit."""
    reqs = make_requests(assets, seed=9, n=24)
    ref = run_alone(vbt, cuda, assets, reqs)
    srv = vbt.Server(hbm_budget_bytes=256 << 20, slots=4)
    ids = [srv.add_asset(a) for a in assets]
    keep, tickets = [], []
    for j, r in enumerate(reqs):
        kind, i, arg = r
        out = cuda.empty(max(out_size(assets[i], r), 1), dtype=cuda.float32, device="cuda")
        if kind == "points":
            q = cuda.from_numpy(arg.view(np.int32)).to("cuda")   # the same bits, in device memory
            tickets.append(srv.submit_points(ids[i], q, out))
            keep.append((q, out))
        elif kind == "slice":
            tickets.append(srv.submit_slice(ids[i], arg[0], arg[1], arg[2], out))
            keep.append((out,))
        else:
            tickets.append(srv.submit_frames(ids[i], arg, out))
            keep.append((out,))
    for j, t in enumerate(tickets):
        res = srv.wait(t)
        assert res.status == 0, (reqs[j][0], res.status)
        srv.release(t)
        got = keep[j][-1][:len(ref[j])].cpu().numpy()
        assert np.array_equal(got.view(np.uint32), ref[j].view(np.uint32)), (j, reqs[j][0])
    srv.close()


@pytest.mark.parametrize("separate", [False, True], ids=["mixed", "separate_kinds"])
def test_mixed_launch_equals_alone(vbt, cuda, assets, separate):
    """Points, slices and frames over several assets, pending together behind a long request, go
    out together: the points in one multi-asset point launch, the slices and frames in one
    persistent mixed launch (serve_mixed_kernel, replayed from the stream's graph) -- far fewer
    units than requests, at most two launches per unit.  Every result equals the plain server's (each
    request on its own kind's kernel) bit for bit; so does the schedule that merges only points."""
    reqs = make_requests(assets, seed=21, n=40)
    alone = run_alone(vbt, cuda, assets, reqs)
    srv = vbt.Server(hbm_budget_bytes=512 << 20, slots=1, separate_kinds=separate)
    ids = [srv.add_asset(a) for a in assets]
    big = assets[0]
    X, Y, Z = big.dims
    n = 1 << 21
    r0 = np.random.default_rng(5)
    hq = np.stack([r0.integers(0, X, n), r0.integers(0, Y, n), r0.integers(0, Z, n),
                   r0.integers(0, big.frames, n)], axis=1).astype(np.uint32)
    hold = srv.submit_points(ids[0], hq, np.empty(n, np.float32))   # pageable: staged by the scheduler
    bufs = [pinned_empty(cuda, out_size(assets[r[1]], r)) for r in reqs]
    tickets = [submit(srv, ids, r, bufs[j][1]) for j, r in enumerate(reqs)]
    assert srv.wait(hold).status == 0
    srv.release(hold)
    for j, t in enumerate(tickets):
        res = srv.wait(t)
        assert res.status == 0, (reqs[j][0], res.status)
        srv.release(t)
    st = srv.stats()
    srv.close()
    for j, r in enumerate(reqs):
        assert np.array_equal(bufs[j][1].view(np.uint32), alone[j].view(np.uint32)), (j, r[0])
    if not separate:
        assert st.units < len(reqs) // 2, st.units
        assert st.launches <= 2 * st.units, (st.launches, st.units)   # points + one mixed launch
