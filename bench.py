#!/usr/bin/env python3
"""Benchmark: decoded voxels/s of the VBTPACK4 temporal decode path on B200.

Workload (the sparse-smoke configuration): a seeded 256^3 x 96 density plume (fBm inside a
rising cone, ~12% of 8^3 leaves non-EMPTY), encoded by the reference encoder
(tests/golden/make_assets.py cfg2_plume).  One step = one pass over the whole 96-frame timeline:
the active-leaf page table is rebuilt from the per-leaf table that the payload walker made when
the asset was uploaded (kernel a), then the current-frame voxel cache (512 FP32 per active leaf) is decoded for every frame (kernel b,
48 frames per launch), into a 96-frame cache ring larger than L2.  L2 is flushed (256 MiB
write) before every timed step.  `value` counts decoded cache voxels (active leaves x 512 x
frames) per second of device time, max over ranks; `e2e` is the same through the C-ABI with host
buffers: the file image is re-uploaded from pinned memory and the whole cache ring is read back.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one per GPU, launched by torchrun); the decode path has no
exchange step, so there is no data-path collective.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DEFAULT_ASSET = os.path.join(ROOT, "assets", "cfg2_plume.vbtp")
WORKLOAD = "sparse smoke plume 256^3 x 96 (cfg2): page table + current-frame cache for all 96 frames per step"
METRIC = "decoded voxels/s"
CHUNK = 48


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=300)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--asset", default=DEFAULT_ASSET)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--no-window", action="store_true")
    p.add_argument("--no-full-frame", action="store_true")
    p.add_argument("--no-sampler", action="store_true")
    p.add_argument("--no-keyframes", action="store_true")
    p.add_argument("--no-writer", action="store_true")
    p.add_argument("--serve-requests", type=int, default=300)
    p.add_argument("--no-ref-queries", action="store_true")
    p.add_argument("--full-size", action="store_true",
                   help="also encode and decode configurations 3 and 4 at their stated sizes (several minutes)")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


# ------------------------------------------------------------------------------ helpers
def max_over_ranks(value, dist, device):
    """The largest `value` over all ranks of the process group (every rank gets it); the plain
    value when there is no group.  Device timings of a multi-GPU step are reported this way."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def algorithmic_bytes_per_frame(rows):
    """Algorithmic bytes of one frame of cache decode for the active leaves of a leaf table:
    8 (header + prefix) + per decoded control 4 desc + 2 bin bytes + 2 keyframes x stride
    + 80 occupancy bytes for Mode2 + 2048 bytes of cache written (512 FP32)."""
    hdr = rows[:, 1]
    info = rows[:, 7]
    active = (info & (1 << 10)) != 0
    hdr, info = hdr[active], info[active]
    mode = hdr & 3
    cc, fcd = (hdr >> 2) & 3, (hdr >> 4) & 3
    cres, fres = (hdr >> 6) & 7, (hdr >> 9) & 7
    cstride = np.where(cc == 1, 8, 3)
    fstride = np.where(fcd == 1, 8, 3)
    fine = (info & (1 << 11)) != 0
    shell = (info & (1 << 12)) != 0
    b = 8 + cres.astype(np.int64) ** 3 * (6 + 2 * cstride)
    b += np.where(fine, fres.astype(np.int64) ** 3 * (6 + 2 * fstride), 0)
    b += np.where(shell, (info & 0x3FF).astype(np.int64) * (6 + 2 * fstride), 0)
    b += np.where(mode == 2, 80, 0)
    b += 2048
    return int(b.sum()), int(active.sum())


class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        """nvidia-smi every 50 ms; each line is stamped with the host clock when it arrives."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True, bufsize=1)
        except Exception:
            self.proc = None
            return

        def reader():
            for line in self.proc.stdout:
                self.lines.append((time.time(), line))

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()
        t0 = time.time()
        while not self.lines and time.time() - t0 < 10.0:   # nvidia-smi takes a moment to start
            time.sleep(0.05)

    def stop(self, t0, t1):
        """Samples that arrived inside the host-clock window [t0, t1] of the timed region."""
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "samples": 0, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, line in list(self.lines):
            if ts < t0 or ts > t1:
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, STREAM-style copy)"
    return 6650.0, "fallback 6.65 TB/s"


def ncu_traffic(frames_per_launch):
    """Per-launch DRAM bytes (read + write) of the decode kernel from the committed ncu summary
    (profiles/decode_leaf_cfg2.md, lines `traffic_bytes_per_launch: N` and
    `traffic_frames_per_launch: F`), if present and captured on launches of this run's shape."""
    p = os.path.join(ROOT, "profiles", "decode_leaf_cfg2.md")
    if not os.path.exists(p):
        return None
    vals = {}
    for line in open(p):
        for key in ("traffic_bytes_per_launch", "traffic_frames_per_launch"):
            if line.startswith(key + ":"):
                vals[key] = int(line.split(":")[1])
    if vals.get("traffic_frames_per_launch") != frames_per_launch:
        return None
    return vals.get("traffic_bytes_per_launch")


# ------------------------------------------------------------------------------ CPU baseline
class CpuDecoder:
    """The cache workload on the host cores: the reference decoder compiled from its sources
    (oracle/_ref, kind "reference") when present, else the C restatement (kind "port")."""

    def __init__(self, asset_path, threads=None):
        import ctypes as C
        from oracle import oracle as orc
        self.cores = threads or os.cpu_count() or 1
        self.f = orc.Oracle().load(asset_path)
        self.compact, self.n_active = self.f.page_table()
        self.frames = self.f.frames
        self.cache = np.zeros(max(self.n_active, 1) * 512, np.float32)
        if os.path.exists(orc.REF_SO):
            self.ref = orc.Reference()
            self.ref.lib.vr_decode_cache.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int]
            self.h = self.ref.load(asset_path)
            self.kind = "reference"
        else:
            self.ref = None
            self.kind = "port"
        self._C, self._orc = C, orc

    def frame(self, t):
        if self.ref is not None:
            if self.ref.lib.vr_decode_cache(self.h, t, self.cache.ctypes.data, self.cores) != 0:
                raise RuntimeError(self.ref.error())
        else:
            C, orc = self._C, self._orc
            self.f.o.lib.vo_decode_cache(C.byref(self.f.f), t, self.compact.ctypes.data_as(orc.u32p),
                                         self.cache.ctypes.data_as(orc.f32p), self.cores)

    def rate(self, seconds):
        """Decode consecutive frames until `seconds` elapse; (voxels/s, sample description)."""
        self.frame(0)
        done, t0 = 0, time.perf_counter()
        while True:
            self.frame(done % self.frames)
            done += 1
            el = time.perf_counter() - t0
            if el >= seconds or done >= 4 * self.frames:
                break
        return (self.n_active * 512 * done / el,
                f"{done} frames of the {self.frames}-frame cache decode ({self.n_active} active leaves), {el:.1f} s")


# ------------------------------------------------------------------------------ serving
SERVE_ASSETS = ["cfg2_plume", "mix_fire_density", "mix_fire_flames", "mix_fire_temperature", "mix_sdf",
                "cfg1_blobs", "cfg4_sdf_small", "mix_sci"]
SERVE_BUDGET = 8 << 30


def serving_requests(assets, n, seed=11):
    """The serving mix: 70% point batches of 1e3..1e6 uniform (x, y, z, t) (log-uniform sizes),
    20% z-slices over 1..16 frames, 10% single dense frames, each on a uniformly drawn asset."""
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n):
        i = int(rng.integers(len(assets)))
        X, Y, Z = assets[i].dims
        T = assets[i].frames
        u = rng.random()
        if u < 0.7:
            m = int(10 ** rng.uniform(3.0, 6.0))
            q = np.empty((m, 4), np.uint32)
            q[:, 0] = rng.integers(0, X, m)
            q[:, 1] = rng.integers(0, Y, m)
            q[:, 2] = rng.integers(0, Z, m)
            q[:, 3] = rng.integers(0, T, m)
            reqs.append(("points", i, q))
        elif u < 0.9:
            t0 = int(rng.integers(0, T))
            reqs.append(("slice", i, (int(rng.integers(0, Z)), t0, min(T, t0 + int(rng.integers(1, 17))))))
        else:
            reqs.append(("frames", i, [int(rng.integers(0, T))]))
    return reqs


def serve_once(vbt, assets, reqs, pinned, plain, arrivals, separate_kinds=False):
    """Run the request list through one server; arrivals=None submits everything at once.
    Latency = done - submit on the server's clock."""
    srv = vbt.Server(hbm_budget_bytes=SERVE_BUDGET, slots=4, plain=plain, host_staging_bytes=256 << 20,
                     separate_kinds=separate_kinds)
    ids = [srv.add_asset(a) for a in assets]
    tickets = [None] * len(reqs)
    t0 = time.perf_counter()
    for j, (kind, i, arg) in enumerate(reqs):
        if arrivals is not None:
            while time.perf_counter() - t0 < arrivals[j]:
                pass
        if kind == "points":
            tickets[j] = srv.submit_points(ids[i], pinned[j][0], pinned[j][1])
        elif kind == "slice":
            tickets[j] = srv.submit_slice(ids[i], *arg)
        else:
            tickets[j] = srv.submit_frames(ids[i], arg)
    lat, first, last, bad = [], None, 0.0, 0
    by_kind = {"points": [], "slice": [], "frames": []}
    for j, t in enumerate(tickets):
        r = srv.wait(t)
        bad += int(r.status != 0)
        lat.append(r.done_ms - r.submit_ms)
        by_kind[reqs[j][0]].append(r.done_ms - r.submit_ms)
        first = r.submit_ms if first is None else min(first, r.submit_ms)
        last = max(last, r.done_ms)
        srv.release(t)
    st = srv.stats()
    srv.close()
    dims = [a.dims for a in assets]
    pts = sum(x[2].shape[0] for x in reqs if x[0] == "points")
    vox = sum((x[2][2] - x[2][1]) * dims[x[1]][0] * dims[x[1]][1] for x in reqs if x[0] == "slice")
    vox += sum(len(x[2]) * dims[x[1]][0] * dims[x[1]][1] * dims[x[1]][2] for x in reqs if x[0] == "frames")
    span_s = (last - first) * 1e-3
    lat = np.array(lat)
    return {"errors": bad, "makespan_ms": last - first, "requests_per_s": len(reqs) / span_s,
            "decoded_values_per_s": (pts + vox) / span_s, "queries_per_s": pts / span_s, "voxels_per_s": vox / span_s,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "p50_p99_ms_by_kind": {k: [float(np.percentile(v, 50)), float(np.percentile(v, 99))]
                                   for k, v in by_kind.items() if v},
            "launches": int(st.launches), "units": int(st.units), "arena_peak_bytes": int(st.arena_peak_bytes)}


def equal_p99_sweep(vbt, assets, reqs, inputs, at_rate, plain_capacity, served_capacity, repeats=3, steps=7):
    """Throughput of served and plain at equal p99.  The target p99 is plain's own at 0.8x its
    closed-loop capacity (median of `repeats` runs), and plain's throughput at that p99 is the rate
    it sustains there.  For the served path, the highest Poisson arrival rate whose median p99 over
    `repeats` runs stays within the target is found by geometric bisection (`steps` halvings
    between 0.25x plain's capacity and 1.5x its own); its throughput at equal p99 is the rate it
    then sustains.  (Searching plain's rate the same way would only re-find 0.8x its capacity,
    and on mixes whose p99 is set by the largest requests' own service time its p99 barely
    depends on the rate, so the search would be noise.)"""
    def p99_at(plain, rate):
        runs = [serve_once(vbt, assets, reqs, inputs, plain, at_rate(rate)) for _ in range(repeats)]
        runs.sort(key=lambda r: r["p99_ms"])
        return runs[len(runs) // 2]

    ref = p99_at(True, 0.8 * plain_capacity)
    target = ref["p99_ms"]
    out = {"target_p99_ms": target, "sweep": {"plain": [{"rate_req_per_s": 0.8 * plain_capacity, "p50_ms": ref["p50_ms"],
                                                          "p99_ms": ref["p99_ms"],
                                                          "achieved_req_per_s": ref["requests_per_s"]}]}}
    best = {"plain": ref["requests_per_s"]}
    for name, plain, cap in (("served", False, served_capacity),):
        lo, hi = 0.25 * plain_capacity, 1.5 * cap
        rows, ok = [], None
        r = p99_at(plain, lo)
        rows.append({"rate_req_per_s": lo, "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"],
                     "achieved_req_per_s": r["requests_per_s"]})
        if r["p99_ms"] <= target:
            ok = r
            for _ in range(steps):
                mid = (lo * hi) ** 0.5
                r = p99_at(plain, mid)
                rows.append({"rate_req_per_s": mid, "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"],
                             "achieved_req_per_s": r["requests_per_s"]})
                if r["p99_ms"] <= target:
                    lo, ok = mid, r
                else:
                    hi = mid
        out["sweep"][name] = sorted(rows, key=lambda x: x["rate_req_per_s"])
        best[name] = ok["requests_per_s"] if ok else 0.0
    out.update({"plain_req_per_s_at_target": best["plain"], "served_req_per_s_at_target": best["served"],
                "throughput_ratio_at_equal_p99": best["served"] / best["plain"] if best["plain"] > 0 else None})
    return out


def pcie_h2d_gbs(local_rank, nbytes=256 << 20, reps=5):
    """Host-to-device copy bandwidth from pinned memory on this box (GB/s, device time)."""
    import torch
    h = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d = torch.empty(nbytes, dtype=torch.uint8, device=f"cuda:{local_rank}")
    d.copy_(h, non_blocking=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        d.copy_(h, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    return nbytes * reps / (e0.elapsed_time(e1) * 1e-3) / 1e9


def encode_mix_asset(vbt, name, local_rank):
    """A render-temporal mix asset that is not on disk, made here: its recipe (tests/golden/
    make_assets.py FIELDS: fire or level set, with its sizes and seed) generated on the GPU
    (tests/golden/gpu_fields.py) and encoded by this library's encoder chain.  Same recipe and size
    as the reference-encoded file; the field's arithmetic is the GPU's, so the bytes may differ."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import gpu_fields as gf
    from make_assets import FIELDS
    from vbt_b200.encode import encode_render_temporal, file_image
    fn, args, index, dims, levelset = FIELDS[name]
    dev = f"cuda:{local_rank}"
    if fn == "fire":
        src = gf.Fire(torch, *args, device=dev)
        slab = lambda z0, z1: src.slab(index, z0, z1)  # noqa: E731
    elif fn == "sdf_scene":
        slab = gf.LevelSet(torch, *args, device=dev).slab
    else:
        return None
    h, off, pay = encode_render_temporal(slab, dims, levelset=levelset)
    img = file_image(h, off, pay)
    del off, pay
    return vbt.Asset(data=img, device=local_rank)


def open_assets(vbt, names, local_rank):
    """The named assets of assets/ that exist, the render-temporal mix assets that do not encoded
    on the GPU from their recipes (encode_mix_asset), and the names skipped, with the reason."""
    assets, opened, skipped = [], [], []
    for n in names:
        p = os.path.join(ROOT, "assets", n + ".vbtp")
        if not os.path.exists(p):
            try:
                a = encode_mix_asset(vbt, n, local_rank)
            except (KeyError, ImportError) as e:
                a = None
                skipped.append(f"{n}: not generated ({e})")
            if a is not None:
                assets.append(a)
                opened.append(n + " (encoded on the GPU from its recipe)")
            elif not skipped or not skipped[-1].startswith(n):
                skipped.append(f"{n}: not generated")
            continue
        try:
            assets.append(vbt.Asset(p, device=local_rank))
            opened.append(n)
        except vbt.VbtError as e:
            skipped.append(f"{n}: {e}")
    return assets, opened, skipped


def run_serving(args, local_rank, assets=None, names=None):
    """The serving mix over the resident assets: served (4 streams, HBM-budget admission, point
    requests merged across assets) against plain (one request per launch, one launch in flight),
    closed loop (all requests at once) and open loop (Poisson arrivals at a common rate).  By
    default the reduced-size mix of assets/; `assets` (open, with their names) replaces it."""
    import torch
    import vbt_b200 as vbt
    own = assets is None
    skipped = []
    if own:
        assets, names, skipped = open_assets(vbt, SERVE_ASSETS, local_rank)
    if len(assets) < 2:
        return {"skipped": "serving-mix assets not generated (tests/golden/make_assets.py)"}
    reqs = serving_requests(assets, args.serve_requests)
    pinned = {}
    for j, (kind, i, arg) in enumerate(reqs):
        if kind == "points":
            q = torch.from_numpy(arg).pin_memory()
            o = torch.empty(arg.shape[0], dtype=torch.float32).pin_memory()
            pinned[j] = (q.numpy(), o.numpy(), q, o)
    serve_once(vbt, assets, reqs[:20], pinned, False, None)   # warm-up
    closed_s = serve_once(vbt, assets, reqs, pinned, False, None)
    closed_p = serve_once(vbt, assets, reqs, pinned, True, None)
    closed_sep = serve_once(vbt, assets, reqs, pinned, False, None, separate_kinds=True)
    gaps = np.random.default_rng(5).exponential(1.0, len(reqs))

    def at_rate(rate):
        return np.cumsum(gaps / rate) - gaps[0] / rate

    lam_p = 0.8 * closed_p["requests_per_s"]
    lam_s = 0.8 * closed_s["requests_per_s"]
    open_s_p = serve_once(vbt, assets, reqs, pinned, False, at_rate(lam_p))
    open_p_p = serve_once(vbt, assets, reqs, pinned, True, at_rate(lam_p))
    open_s_s = serve_once(vbt, assets, reqs, pinned, False, at_rate(lam_s))
    # the same requests from a client that keeps its query batches and results on the GPU (a
    # renderer): point inputs in device memory, every result device-resident
    dev = {j: (torch.from_numpy(arg.view(np.int32)).to(f"cuda:{local_rank}"), None)
           for j, (kind, i, arg) in enumerate(reqs) if kind == "points"}
    serve_once(vbt, assets, reqs[:20], dev, False, None)   # warm-up
    d_closed_s = serve_once(vbt, assets, reqs, dev, False, None)
    d_closed_p = serve_once(vbt, assets, reqs, dev, True, None)
    d_lam_p = 0.8 * d_closed_p["requests_per_s"]
    d_lam_s = 0.8 * d_closed_s["requests_per_s"]
    d_open_s_p = serve_once(vbt, assets, reqs, dev, False, at_rate(d_lam_p))
    d_open_p_p = serve_once(vbt, assets, reqs, dev, True, at_rate(d_lam_p))
    d_open_s_s = serve_once(vbt, assets, reqs, dev, False, at_rate(d_lam_s))
    equal_host = equal_p99_sweep(vbt, assets, reqs, pinned, at_rate, closed_p["requests_per_s"],
                                 closed_s["requests_per_s"])
    equal_dev = equal_p99_sweep(vbt, assets, reqs, dev, at_rate, d_closed_p["requests_per_s"],
                                d_closed_s["requests_per_s"])
    if own:
        for a in assets:
            a.close()
    # the PCIe bound of the host-buffer mix: its point queries in (16 B each) and values out (4 B)
    h2d = pcie_h2d_gbs(local_rank)
    q_in = sum(16 * r[2].shape[0] for r in reqs if r[0] == "points")
    pcie_ms = q_in / (h2d * 1e9) * 1e3
    pcie = {"h2d_gbs_pinned": h2d, "point_input_bytes": q_in,
            "point_output_bytes": sum(4 * r[2].shape[0] for r in reqs if r[0] == "points"),
            "min_makespan_ms_from_h2d": pcie_ms, "max_req_per_s_from_h2d": len(reqs) / (pcie_ms * 1e-3),
            "bound_vs_plain_closed_loop": (len(reqs) / (pcie_ms * 1e-3)) / closed_p["requests_per_s"]}
    return {"workload": "serving mix: 70% point batches of 1e3-1e6 uniform (x,y,z,t), 20% z-slices over 1-16 "
                        "frames, 10% dense frames, uniform over the assets; point inputs and outputs in pinned host "
                        "memory, slice and frame results device-resident (released when done)",
            "assets": names, "assets_skipped": skipped, "requests": len(reqs),
            "kinds": {k: sum(1 for r in reqs if r[0] == k) for k in ("points", "slice", "frames")},
            "server": {"hbm_budget_bytes": SERVE_BUDGET, "slots": 4},
            "served": {"closed_loop": closed_s, "poisson_at_0.8x_plain_capacity": open_s_p,
                       "poisson_at_0.8x_served_capacity": open_s_s},
            "served_separate_kinds": {"closed_loop": closed_sep,
                                      "note": "points merged, each slice and frame on its own kernel"},
            "plain": {"closed_loop": closed_p, "poisson_at_0.8x_plain_capacity": open_p_p},
            "throughput_ratio_closed_loop": closed_s["decoded_values_per_s"] / closed_p["decoded_values_per_s"],
            "equal_p99": equal_host, "pcie_bound": pcie,
            "arrival_rates_req_per_s": {"0.8x_plain": lam_p, "0.8x_served": lam_s},
            "device_resident": {
                "workload": "the same requests with point inputs in device memory and every result device-resident",
                "served": {"closed_loop": d_closed_s, "poisson_at_0.8x_plain_capacity": d_open_s_p,
                           "poisson_at_0.8x_served_capacity": d_open_s_s},
                "plain": {"closed_loop": d_closed_p, "poisson_at_0.8x_plain_capacity": d_open_p_p},
                "throughput_ratio_closed_loop": d_closed_s["decoded_values_per_s"] / d_closed_p["decoded_values_per_s"],
                "equal_p99": equal_dev,
                "arrival_rates_req_per_s": {"0.8x_plain": d_lam_p, "0.8x_served": d_lam_s}}}


# ------------------------------------------------------------------------------ full frames
def run_full_frame(args, local_rank, a, rows, reps=5):
    """Dense full-frame decode (vbt_decode_frames, 48 frames per launch) of the bench asset:
    every voxel of every frame written, EMPTY leaves as zeros.  Algorithmic bytes per frame =
    the active leaves' decode bytes (as the cache workload, less the 2 KiB cache write per leaf)
    + 4 X Y Z bytes of frame written."""
    import torch
    X, Y, Z = a.dims
    T = a.frames
    fpl = min(48, T)
    vox = X * Y * Z
    out = torch.empty((fpl, vox), dtype=torch.float32, device=f"cuda:{local_rank}")
    bytes_cache, n_act = algorithmic_bytes_per_frame(rows)
    per_frame = bytes_cache - 2048 * n_act + 4 * vox
    s = torch.cuda.Stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    with torch.cuda.stream(s):
        a.decode_frames(list(range(fpl)), out, stream=s)
        for k, (e0, e1) in enumerate(ev):
            f0 = (k * fpl) % max(1, T - fpl + 1)
            e0.record(s)
            a.decode_frames(list(range(f0, f0 + fpl)), out, stream=s)
            e1.record(s)
    s.synchronize()
    a.sync_status(s)
    ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)
    peak, _ = measured_peak()
    gbs = per_frame * fpl / (ms * 1e-3) / 1e9
    return {"frames_per_launch": fpl, "ms_per_launch": ms, "voxels_per_s": vox * fpl / (ms * 1e-3),
            "algorithmic_bytes_per_frame": per_frame, "achieved_gbs": gbs, "frac_of_measured_hbm": gbs / peak,
            "output_bytes_per_launch": 4 * vox * fpl,
            "note": "output larger than L2; consecutive launches write the same 48-frame buffer"}


# ------------------------------------------------------------------------------ (d) precision
WINDOW_ASSET = os.path.join(ROOT, "assets", "mix_sci.vbtp")


def run_window(args, local_rank, reps=10):
    """(d) on the scientific field (config-5 scene, 128^3 x 64): the whole 64-frame timeline as
    one tensor-core window per leaf (vbt_decode_window) against the exact per-frame decode of the
    same frames (vbt_decode_cache, 64 frames per launch); device time per timeline, and the error
    of both against the FP64 oracle, relative to the field range."""
    import torch
    import vbt_b200 as vbt
    path = WINDOW_ASSET if os.path.exists(WINDOW_ASSET) else os.path.join(ROOT, "assets", "sci_64.vbtp")
    if not os.path.exists(path):
        return {"skipped": "no scientific asset generated"}
    a = vbt.Asset(path, device=local_rank)
    T, L = a.frames, a.leaf_count
    n = min(T, 64)
    s = torch.cuda.Stream()
    win = torch.empty((n, L, 512), dtype=torch.float32, device=f"cuda:{local_rank}")
    ref = torch.empty_like(win)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=win.device)

    def timed(fn):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        with torch.cuda.stream(s):
            fn()
            for e0, e1 in ev:
                flush.zero_()
                e0.record(s)
                fn()
                e1.record(s)
        s.synchronize()
        return statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)

    win_ms = timed(lambda: a.decode_window(0, n, win, stream=s))
    ref_ms = timed(lambda: a.decode_cache(list(range(n)), ref, frame_stride=L * 512, stream=s))
    a.sync_status(s)
    mx_w, rms_w, lo, hi = a.window_error(0, n, win, stream=s)
    mx_r, rms_r, _, _ = a.window_error(0, n, ref, stream=s)
    rng = hi - lo
    vox = L * 512 * n
    a.close()
    return {"asset": os.path.basename(path), "frames": n, "leaves": L,
            "tensor_core_window": {"ms_per_timeline": win_ms, "voxels_per_s": vox / (win_ms * 1e-3),
                                   "max_abs_err_rel_range": mx_w / rng, "rms_err_rel_range": rms_w / rng,
                                   "products": "split-BF16: exact S' x three BF16 terms of C, FP32 accumulate"},
            "fp32_per_frame": {"ms_per_timeline": ref_ms, "voxels_per_s": vox / (ref_ms * 1e-3),
                               "max_abs_err_rel_range": mx_r / rng, "rms_err_rel_range": rms_r / rng},
            "oracle": "FP64 on the GPU (reference model without intermediate rounding), range "
                      f"{lo:.6g} .. {hi:.6g}", "speedup": ref_ms / win_ms}


RENDER_WINDOW_ASSETS = ["mix_fire_density", "mix_fire_flames", "mix_fire_temperature"]


def run_window_render(args, local_rank, reps=5):
    """(d) on the fire (config-3 scene, three fields 128 x 128 x 192 x 40): 16-frame timeline
    windows per active leaf (vbt_decode_window: exact voxels at the union of key-frame knots, hat
    basis x knot coefficients on the tensor cores) over the whole timeline, against the exact
    per-frame decode of the same frames (vbt_decode_cache, 16 frames per launch); device time and
    the error of both against the FP64 oracle, relative to each field's range."""
    import torch
    import vbt_b200 as vbt
    out = {}
    for name in RENDER_WINDOW_ASSETS:
        path = os.path.join(ROOT, "assets", name + ".vbtp")
        if not os.path.exists(path):
            continue
        a = vbt.Asset(path, device=local_rank)
        a.build_page_table()
        T, A = a.frames, a.active_count
        W = 16
        starts = list(range(0, T - W + 1, W))
        n = len(starts) * W
        s = torch.cuda.Stream()
        win = torch.empty((n, A, 512), dtype=torch.float32, device=f"cuda:{local_rank}")
        ref = torch.empty_like(win)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=win.device)

        def timed(fn):
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
            with torch.cuda.stream(s):
                fn()
                for e0, e1 in ev:
                    flush.zero_()
                    e0.record(s)
                    fn()
                    e1.record(s)
            s.synchronize()
            return statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)

        win_ms = timed(lambda: [a.decode_window(t, W, win[t], frame_stride=A * 512, stream=s) for t in starts])
        ref_ms = timed(lambda: [a.decode_cache(list(range(t, t + W)), ref[t], frame_stride=A * 512, stream=s)
                                for t in starts])
        a.sync_status(s)
        mx_w, rms_w, lo, hi = a.window_error(0, n, win, frame_stride=A * 512, stream=s)
        mx_r, rms_r, _, _ = a.window_error(0, n, ref, frame_stride=A * 512, stream=s)
        rng = hi - lo
        vox = A * 512 * n
        out[name] = {"frames": n, "windows": len(starts), "active_leaves": A,
                     "tensor_core_window": {"ms": win_ms, "voxels_per_s": vox / (win_ms * 1e-3),
                                            "max_abs_err_rel_range": mx_w / rng, "rms_err_rel_range": rms_w / rng},
                     "fp32_per_frame": {"ms": ref_ms, "voxels_per_s": vox / (ref_ms * 1e-3),
                                        "max_abs_err_rel_range": mx_r / rng, "rms_err_rel_range": rms_r / rng},
                     "oracle_range": [lo, hi], "speedup": ref_ms / win_ms}
        a.close()
    if not out:
        return {"skipped": "no fire assets generated"}
    out["products"] = "hat basis H(16 x K) x exact knot voxels, both split into three BF16 terms, FP32 accumulate"
    return out


# ------------------------------------------------------------------------------ ray sampler
def camera_rays(dims, width, height, fov_deg=40.0):
    """A pinhole camera outside the volume looking at its centre: rays [width * height, 8] float32
    (origin, t_min = 0, direction, t_max), each starting where it enters the volume's box and
    ending where it leaves it (t_max = 0 for rays that miss), as a ray generator hands them over."""
    X, Y, Z = dims
    centre = np.array([X / 2.0, Y / 2.0, Z / 2.0])
    eye = centre + np.array([0.35 * X, -1.6 * Y, 0.45 * Z])
    fwd = centre - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, [0.0, 0.0, 1.0])
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    h = np.tan(np.radians(fov_deg) / 2.0)
    u = (np.arange(width) + 0.5) / width * 2.0 - 1.0
    v = (np.arange(height) + 0.5) / height * 2.0 - 1.0
    uu, vv = np.meshgrid(u * h * width / height, v * h)
    d = fwd[None, None, :] + uu[..., None] * right + vv[..., None] * up
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    d = d.reshape(-1, 3)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / d
        t0 = (np.zeros(3) - eye) * inv
        t1 = (np.array([X - 1.0, Y - 1.0, Z - 1.0]) - eye) * inv
    near = np.maximum(np.minimum(t0, t1).max(axis=1), 0.0)
    far = np.maximum(t0, t1).min(axis=1)
    hit = far > near
    rays = np.zeros((height * width, 8), np.float32)
    rays[:, 0:3] = eye + d * np.where(hit, near, 0.0)[:, None]
    rays[:, 4:7] = d
    rays[:, 7] = np.where(hit, far - near, 0.0)
    return rays


def run_sampler(args, local_rank, reps=5):
    """Ray sampling from the control cache (vbt_sample_rays; the Studio's vbt_sample.comp) on one
    B200: a 1920 x 1080 pinhole view of the plume (density accumulation, 256 steps per ray) and of
    the level set (surface tracing with thickness and floor shadow, up to 160 steps), one frame's
    control cache built first.  Rays/s and samples/s of device time, beside the C restatement of
    the shader (the oracle) on the host threads for a bounded sample of the same rays."""
    import torch
    import vbt_b200 as vbt
    from oracle.oracle import Oracle, VoSampleParams
    scenes = [("cfg2_plume", 0, 256, 0), ("mix_sdf", 1, 160, 1)]
    out = {}
    orc = None
    for name, mode, steps, model in scenes:
        path = os.path.join(ROOT, "assets", name + ".vbtp")
        if not os.path.exists(path):
            continue
        a = vbt.Asset(path, device=local_rank)
        a.build_page_table()
        frame = a.frames // 2
        n_act = a.active_count
        dev = f"cuda:{local_rank}"
        ctrl = torch.empty((1, max(n_act, 1), 576), dtype=torch.float32, device=dev)
        rays = camera_rays(a.dims, 1920, 1080)
        d_rays = torch.from_numpy(rays).to(dev)
        res = torch.empty_like(d_rays)
        p = vbt.SampleParams()
        p.step_count, p.frame_index, p.render_mode, p.voxel_size = steps, frame, mode, 1.0
        p.background_value = 1.0 if mode == 1 else 0.0
        p.surface_iso, p.surface_epsilon_voxels, p.surface_normal_step, p.max_step_voxels = 0.0, 0.5, 1.0, 4.0
        p.surface_model, p.floor_height, p.shadow_steps, p.up_axis = model, 1.0, 48, 2
        s = torch.cuda.Stream(device=dev)
        s.wait_stream(torch.cuda.current_stream(dev))      # the rays were copied on the current stream
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
               torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        with torch.cuda.stream(s):
            a.decode_control_cache([frame], ctrl, frame_stride=max(n_act, 1) * 576, stream=s)
            a.sample_rays(ctrl, p, d_rays, res, stream=s)
            for e0, e1, e2 in ev:
                e0.record(s)
                a.decode_control_cache([frame], ctrl, frame_stride=max(n_act, 1) * 576, stream=s)
                e1.record(s)
                a.sample_rays(ctrl, p, d_rays, res, stream=s)
                e2.record(s)
        s.synchronize()
        a.sync_status(s)
        cache_ms = statistics.mean(e0.elapsed_time(e1) for e0, e1, _ in ev)
        ray_ms = statistics.mean(e1.elapsed_time(e2) for _, e1, e2 in ev)
        n = rays.shape[0]
        entry = {"rays": n, "render_mode": mode, "step_count": steps, "frame": frame,
                 "control_cache_ms": cache_ms, "sample_ms": ray_ms, "rays_per_s": n / (ray_ms * 1e-3)}
        if mode == 0:
            entry["samples_per_s"] = n * steps / (ray_ms * 1e-3)
        else:
            entry["rays_hit"] = int((res[:, 3] >= 0).sum().item())
        # the C restatement on the host threads, on a bounded sample of the rays
        if not args.no_cpu:
            orc = orc or Oracle()
            f = orc.load(path)
            compact, _ = f.page_table()
            cache = f.control_cache(frame, compact)
            q = VoSampleParams()
            for fld, _ in VoSampleParams._fields_:
                if fld != "bbox_min":
                    setattr(q, fld, getattr(p, fld))
            m = 20000 if mode == 0 else 50000
            sample = rays[:: max(1, n // m)][:m]
            t0 = time.perf_counter()
            f.sample_rays(cache, compact, q, sample)
            el = time.perf_counter() - t0
            entry["cpu_restatement"] = {"rays_per_s": sample.shape[0] / el, "cores": os.cpu_count(),
                                        "sample": f"{sample.shape[0]} of the {n} rays"}
        out[name] = entry
        a.close()
    return out or {"skipped": "assets not generated"}


# ------------------------------------------------------------------------------ keyframe pass
def gpu_blobs(shape_xyz, frames, n_blobs, seed, dev, noise=0.01):
    """The config-1 blob recipe (tests/golden/make_assets.py: blobs) evaluated on the GPU: frames
    [T, Z*Y*X] float32, blob parameters from the same seeded draws, the noise from a seeded torch
    generator."""
    import torch
    rng = np.random.default_rng(seed)
    X, Y, Z = shape_xyz
    sig = rng.uniform(4.0, 10.0, n_blobs)
    amp = rng.uniform(0.2, 1.0, n_blobs)
    c0 = rng.uniform(0.2, 0.8, (n_blobs, 3)) * np.array([X, Y, Z])
    d = rng.normal(size=(n_blobs, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    vel = d * rng.uniform(0.0, 1.0, (n_blobs, 1))
    zz, yy, xx = torch.meshgrid(torch.arange(Z, device=dev, dtype=torch.float32),
                                torch.arange(Y, device=dev, dtype=torch.float32),
                                torch.arange(X, device=dev, dtype=torch.float32), indexing="ij")
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    out = torch.empty((frames, Z * Y * X), dtype=torch.float32, device=dev)
    for t in range(frames):
        f = torch.randn((Z, Y, X), generator=gen, device=dev, dtype=torch.float32) * noise
        for b in range(n_blobs):
            c = c0[b] + vel[b] * t
            r2 = (xx - float(c[0])) ** 2 + (yy - float(c[1])) ** 2 + (zz - float(c[2])) ** 2
            f += float(amp[b]) * torch.exp(-r2 / float(2.0 * sig[b] ** 2))
        out[t] = f.reshape(-1)
    return out


def run_keyframes(args, local_rank, reps=3, work=None):
    """The encoder's per-voxel keyframe pass (vbt_detect_keyframes: background test,
    detectDensityKeyFrames, reconstructFromKeys, squared error) on one B200, with the encoder's
    default profile, over (1) the config-1 field itself (64^3 x 24 blobs, tests/golden/
    make_assets.py) and (2) the same recipe at the plume's size, 256^3 x 96, generated on the GPU.
    Device time of the whole pass (inputs resident, outputs: key masks, counts, flags,
    reconstruction, errors, totals); beside it the reference's own detector (oracle/_ref/libkfref.so)
    on all host threads for a bounded sample of the same series, whose key counts are checked
    against the GPU's."""
    import torch
    import vbt_b200 as vbt
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_assets import blobs
    dev = f"cuda:{local_rank}"
    out = {}
    ref = None
    try:
        from oracle.oracle import KeyframeReference, VoKeyframeProfile
        ref = KeyframeReference()
    except (OSError, ImportError):
        pass
    work = work or [("config1_blobs_64^3x24",
                     lambda: torch.from_numpy(blobs((64, 64, 64), 24, 6, 1).reshape(24, -1)).to(dev)),
                    ("blobs_256^3x96", lambda: gpu_blobs((256, 256, 256), 96, 6, 2, dev))]
    prof = vbt.KeyframeProfile()
    for name, make in work:
        frames = make()
        T, S = frames.shape
        W = (T + 31) // 32
        mask = torch.empty((W, S), dtype=torch.int32, device=dev)
        cnt = torch.empty(S, dtype=torch.int32, device=dev)
        flags = torch.empty(S, dtype=torch.uint8, device=dev)
        recon = torch.empty_like(frames)
        err2 = torch.empty(S, dtype=torch.float64, device=dev)
        tot = torch.empty(40, dtype=torch.uint8, device=dev)
        s = torch.cuda.Stream(device=dev)
        s.wait_stream(torch.cuda.current_stream(dev))      # the frames were made on the current stream
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        with torch.cuda.stream(s):
            vbt.detect_keyframes(frames, prof, mask, cnt, flags, recon, err2, tot, stream=s)
            for e0, e1 in ev:
                e0.record(s)
                vbt.detect_keyframes(frames, prof, mask, cnt, flags, recon, err2, tot, stream=s)
                e1.record(s)
        s.synchronize()
        ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)
        t = vbt.keyframe_totals(tot)
        moved = S * T * 4 * 2 + S * (W * 4 + 4 + 1 + 8)
        e2e = None
        if S * T * 4 <= (1 << 30):
            # end to end from pinned host memory: frames in; reconstruction, key masks, counts and
            # flags out, every step
            h_in = frames.cpu().pin_memory()
            h_recon = torch.empty(recon.shape, dtype=recon.dtype).pin_memory()
            h_mask = torch.empty(mask.shape, dtype=mask.dtype).pin_memory()
            h_cnt = torch.empty(cnt.shape, dtype=cnt.dtype).pin_memory()
            h_flags = torch.empty(flags.shape, dtype=flags.dtype).pin_memory()
            ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
            with torch.cuda.stream(s):
                for e0, e1 in ev2:
                    e0.record(s)
                    frames.copy_(h_in, non_blocking=True)
                    vbt.detect_keyframes(frames, prof, mask, cnt, flags, recon, None, None, stream=s)
                    h_recon.copy_(recon, non_blocking=True)
                    h_mask.copy_(mask, non_blocking=True)
                    h_cnt.copy_(cnt, non_blocking=True)
                    h_flags.copy_(flags, non_blocking=True)
                    e1.record(s)
            s.synchronize()
            e2e_ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev2)
            e2e = {"series_per_s": S / (e2e_ms * 1e-3), "ms": e2e_ms, "h2d_bytes": S * T * 4,
                   "d2h_bytes": S * T * 4 + S * (W * 4 + 4 + 1)}
        entry = {"series": S, "frames": T, "pass_ms": ms, "series_per_s": S / (ms * 1e-3),
                 "values_per_s": S * T / (ms * 1e-3), "bytes_moved": moved, "gb_per_s": moved / (ms * 1e-3) / 1e9,
                 "keys_per_series": t.total_keys / S, "max_keys": t.max_keys,
                 "background_series": t.background_series, "protected_series": t.protected_series,
                 "bound": "fp64/integer issue (the pass reads and writes each value once)", "e2e": e2e}
        if ref is not None and not args.no_cpu:
            n = min(S, 65536 if T > 32 else S)
            sample = frames[:, :n].cpu().numpy()
            threads = os.cpu_count()
            t0 = time.perf_counter()
            kc, _ = ref.temporal_pass(sample, VoKeyframeProfile(), threads=threads)
            el = time.perf_counter() - t0
            entry["cpu_reference"] = {"series_per_s": n / el, "cores": threads, "kind": "reference",
                                      "sample": f"the first {n} of {S} series"}
            entry["sample_key_counts_equal"] = bool(np.array_equal(kc, cnt[:n].cpu().numpy().view(np.uint32)))
            entry["speedup_vs_cpu_reference"] = entry["series_per_s"] / entry["cpu_reference"]["series_per_s"]
        out[name] = entry
        del frames, recon, mask
        torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------------------------ reference CUDA queries
REF_QUERY_BENCH = os.path.join(ROOT, "oracle", "_ref", "vbt_cuda_query_bench")
REF_QUERY_ASSETS = ["mix_sci", "sci_modes", "cfg5_sci"]


def run_reference_queries(args, local_rank, n=1_000_000, repeats=100):
    """Scientific point queries on one B200: the reference's own CUDA benchmark
    (render/src/vbt_cuda_query_bench.cu, vbtQueryKernel on the queries as drawn and
    vbtGroupedLeafQueryKernel on them sorted by leaf; built unmodified for sm_100a by
    oracle/Makefile) beside this library's point-query kernel, on the same asset, the same number
    of uniform random (x, y, z, t) queries (the reference's generator and seed on its side, numpy's
    on this one), the same repeat count, device time by CUDA events over the repeats on both
    sides, inputs resident."""
    import tempfile

    import torch
    import vbt_b200 as vbt
    if not os.path.exists(REF_QUERY_BENCH):
        return {"skipped": "oracle/_ref/vbt_cuda_query_bench not built (the reference tree is absent)"}
    out = {}
    dev = f"cuda:{local_rank}"
    for name in REF_QUERY_ASSETS:
        path = os.path.join(ROOT, "assets", name + ".vbtp")
        if not os.path.exists(path):
            continue
        with tempfile.TemporaryDirectory() as td:
            js = os.path.join(td, "ref.json")
            cmd = [REF_QUERY_BENCH, "--input-vbt", path, "--query-count", str(n), "--pattern", "random",
                   "--fixed-frame", "0", "--seed", "7", "--repeats", str(repeats), "--json-out", js]
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
            if r.returncode != 0 or not os.path.exists(js):
                out[name] = {"reference_failed": (r.stderr or r.stdout)[-300:]}
                continue
            ref = json.load(open(js))
        a = vbt.Asset(path, device=local_rank)
        X, Y, Z = a.dims
        T = a.frames
        rng = np.random.default_rng(7)
        q = np.stack([rng.integers(0, X, n), rng.integers(0, Y, n), rng.integers(0, Z, n), rng.integers(0, T, n)],
                     1).astype(np.uint32)
        leaf = ((q[:, 2] // 8) * ((Y + 7) // 8) + q[:, 1] // 8) * ((X + 7) // 8) + q[:, 0] // 8
        q_sorted = q[np.lexsort((q[:, 0], q[:, 1], q[:, 2], q[:, 3], leaf))]
        res = {}
        for label, qq in (("unsorted", q), ("sorted", q_sorted)):
            dq = torch.from_numpy(np.ascontiguousarray(qq).view(np.int32)).to(dev)
            o = torch.empty(n, dtype=torch.float32, device=dev)
            s = torch.cuda.Stream(device=dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s):
                for _ in range(3):
                    a.query_points(dq, o, stream=s)
                e0.record(s)
                for _ in range(repeats):
                    a.query_points(dq, o, stream=s)
                e1.record(s)
            s.synchronize()
            a.sync_status(s)
            ms = e0.elapsed_time(e1)
            res[label] = {"kernel_ms": ms, "queries_per_s": n * repeats / (ms * 1e-3)}
        a.close()
        # the grouped kernel decodes a leaf's controls once, at its first query's frame, for every
        # query of the leaf: on random-t queries it is not the reference's decode (its own check
        # against the reference CPU decoder reports the difference), so the fair best of the
        # reference is its best run whose values agree with the CPU decoder
        tol = 1e-4   # absolute; the fields span about +-15 (the grouped kernel misses by up to ~5)
        ok = {k: ref[k]["max_abs_diff"] <= tol for k in ("unsorted", "sorted")}
        valid = [ref[k]["queries_per_sec"] for k in ("unsorted", "sorted") if ok[k]]
        best_ref = max(valid) if valid else max(ref["unsorted"]["queries_per_sec"], ref["sorted"]["queries_per_sec"])
        out[name] = {"queries": n, "repeats": repeats, "pattern": "uniform random (x, y, z, t)",
                     "reference_cuda": {"unsorted_queries_per_s": ref["unsorted"]["queries_per_sec"],
                                        "sorted_grouped_queries_per_s": ref["sorted"]["queries_per_sec"],
                                        "unsorted_max_abs_diff_vs_reference_cpu": ref["unsorted"]["max_abs_diff"],
                                        "sorted_grouped_max_abs_diff_vs_reference_cpu": ref["sorted"]["max_abs_diff"],
                                        "agrees_with_reference_cpu": ok},
                     "ours": {"unsorted_queries_per_s": res["unsorted"]["queries_per_s"],
                              "sorted_queries_per_s": res["sorted"]["queries_per_s"]},
                     "speedup_unsorted": res["unsorted"]["queries_per_s"] / ref["unsorted"]["queries_per_sec"],
                     "speedup_sorted": res["sorted"]["queries_per_s"] / ref["sorted"]["queries_per_sec"],
                     "speedup_best_vs_best_agreeing": max(res["unsorted"]["queries_per_s"], res["sorted"]["queries_per_s"]) /
                     best_ref}
    return out or {"skipped": "no scientific asset generated"}


# ------------------------------------------------------------------------------ configs 3 and 4 at full size
def timed_ms(torch, s, fn, reps, flush=None):
    """Mean device time (CUDA events on stream s) of fn over reps runs after one untimed run."""
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    with torch.cuda.stream(s):
        fn()
        for e0, e1 in ev:
            if flush is not None:
                flush.zero_()
            e0.record(s)
            fn()
            e1.record(s)
    s.synchronize()
    return statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)


def encode_on_gpu(torch, slab, dims, levelset):
    """A field produced slab by slab on the GPU, encoded there (vbt_b200.encode) and brought into a
    pinned host file image; (image, seconds)."""
    from vbt_b200.encode import encode_render_temporal, file_image
    t0 = time.time()
    h, off, pay = encode_render_temporal(slab, dims, levelset=levelset)
    torch.cuda.synchronize()
    img = file_image(h, off, pay, pinned=True)
    return img, time.time() - t0


def cache_timeline(torch, a, dev, W=16, reps=2):
    """The whole timeline as W-frame cache launches into one W-frame ring: device ms per timeline,
    voxels/s and the fraction of measured HBM peak of the algorithmic bytes."""
    T, A = a.frames, a.active_count
    ring = torch.empty((W, A, 512), dtype=torch.float32, device=dev)
    s = torch.cuda.Stream(device=dev)
    chunks = [list(range(t, min(T, t + W))) for t in range(0, T, W)]
    ms = timed_ms(torch, s, lambda: [a.decode_cache(ch, ring, frame_stride=A * 512, stream=s) for ch in chunks], reps)
    a.sync_status(s)
    per_frame, _ = algorithmic_bytes_per_frame(a.leaf_table())
    peak, _ = measured_peak()
    gbs = per_frame * T / (ms * 1e-3) / 1e9
    del ring
    return {"frames_per_launch": W, "ms_per_timeline": ms, "voxels_per_s": A * 512 * T / (ms * 1e-3),
            "algorithmic_bytes_per_frame": per_frame, "achieved_gbs": gbs, "frac_of_measured_hbm": gbs / peak}


def window_vs_exact(torch, a, dev, W=16):
    """(d) over the whole timeline in W-frame windows per active leaf: the tensor-core window
    (vbt_decode_window) and the exact per-frame decode (vbt_decode_cache), device time of each,
    and the error of each against the FP64 oracle relative to the field's range."""
    T, A = a.frames, a.active_count
    starts = list(range(0, T - W + 1, W))
    win = torch.empty((W, A, 512), dtype=torch.float32, device=dev)
    ref = torch.empty_like(win)
    s = torch.cuda.Stream(device=dev)
    win_ms = timed_ms(torch, s, lambda: [a.decode_window(t, W, win, frame_stride=A * 512, stream=s) for t in starts], 2)
    ref_ms = timed_ms(torch, s, lambda: [a.decode_cache(list(range(t, t + W)), ref, frame_stride=A * 512, stream=s)
                                         for t in starts], 2)
    stats = {"window": [0.0, 0.0], "exact": [0.0, 0.0]}
    lo, hi = float("inf"), float("-inf")
    for t in starts:
        with torch.cuda.stream(s):
            a.decode_window(t, W, win, frame_stride=A * 512, stream=s)
            a.decode_cache(list(range(t, t + W)), ref, frame_stride=A * 512, stream=s)
        for key, buf in (("window", win), ("exact", ref)):
            mx, rms, l, h = a.window_error(t, W, buf, frame_stride=A * 512, stream=s)
            stats[key][0] = max(stats[key][0], mx)
            stats[key][1] += rms * rms
            lo, hi = min(lo, l), max(hi, h)
    a.sync_status(s)
    rng = hi - lo
    vox = A * 512 * W * len(starts)
    del win, ref
    return {"windows": len(starts), "frames": W * len(starts), "oracle_range": [lo, hi],
            "tensor_core_window": {"ms": win_ms, "voxels_per_s": vox / (win_ms * 1e-3),
                                   "max_abs_err_rel_range": stats["window"][0] / rng,
                                   "rms_err_rel_range": (stats["window"][1] / len(starts)) ** 0.5 / rng},
            "fp32_per_frame": {"ms": ref_ms, "voxels_per_s": vox / (ref_ms * 1e-3),
                               "max_abs_err_rel_range": stats["exact"][0] / rng,
                               "rms_err_rel_range": (stats["exact"][1] / len(starts)) ** 0.5 / rng},
            "speedup": ref_ms / win_ms}


def dense_timeline(torch, a, dev, W=16, reps=2):
    """Dense full frames (vbt_decode_frames) over the whole timeline, W frames per launch into one
    W-frame buffer: device ms, voxels/s, and the fraction of measured HBM peak of the algorithmic
    bytes (active leaves' decode bytes, less the cache write, plus 4 bytes per voxel written)."""
    X, Y, Z = a.dims
    T, vox = a.frames, a.dims[0] * a.dims[1] * a.dims[2]
    out = torch.empty((W, vox), dtype=torch.float32, device=dev)
    s = torch.cuda.Stream(device=dev)
    chunks = [list(range(t, min(T, t + W))) for t in range(0, T, W)]
    ms = timed_ms(torch, s, lambda: [a.decode_frames(ch, out, stream=s) for ch in chunks], reps)
    a.sync_status(s)
    bytes_cache, n_act = algorithmic_bytes_per_frame(a.leaf_table())
    per_frame = bytes_cache - 2048 * n_act + 4 * vox
    peak, _ = measured_peak()
    gbs = per_frame * T / (ms * 1e-3) / 1e9
    del out
    return {"frames_per_launch": W, "ms_per_timeline": ms, "voxels_per_s": vox * T / (ms * 1e-3),
            "algorithmic_bytes_per_frame": per_frame, "achieved_gbs": gbs, "frac_of_measured_hbm": gbs / peak}


def run_full_size(args, local_rank):
    """Configurations 3 and 4 at their stated sizes.  The raw fields (36-64 GB of float32 each) are
    generated on the GPU from their seeds (tests/golden/gpu_fields.py), slab by slab, and encoded
    there by this library's encoder chain (vbt_b200.encode; byte-exact against the reference encoder
    on the reduced assets), so no raw field or large asset leaves the box.
      config 3: the fire's three aligned fields, 384 x 384 x 512 x 120: the cache timeline and the
                (d) window decode against the exact decode, with the error against the FP64 oracle;
      config 4: the liquid level set, 512^3 x 120, Mode2 shell: dense full frames over the timeline;
      config 5: the serving mix over eight resident assets of the stated sizes (the five above, the
                plume, the 512^3 x 64 scientific field, and the two small scenes).
    Decoded values are checked against the oracle in tests/test_full_size.py."""
    import torch
    import vbt_b200 as vbt
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import gpu_fields as gf
    dev = f"cuda:{local_rank}"
    out = {}
    resident, names = [], []
    fire = gf.Fire(torch, **gf.FIRE_FULL, device=dev)
    dims = gf.FIRE_FULL["shape_xyz"]
    for i, name in enumerate(("density", "flames", "temperature")):
        img, enc_s = encode_on_gpu(torch, lambda z0, z1: fire.slab(i, z0, z1), dims, False)
        a = vbt.Asset(data=img, device=local_rank)
        a.build_page_table()
        out["config3_fire_" + name] = {
            "dims": list(dims) + [a.frames], "leaves": a.leaf_count, "active_leaves": a.active_count,
            "file_bytes": int(img.numel()), "encode_s": enc_s,
            "cache_timeline": cache_timeline(torch, a, dev), "precision_window": window_vs_exact(torch, a, dev)}
        resident.append(a)
        names.append("config3_fire_" + name)
        del img
    del fire
    torch.cuda.empty_cache()
    lv = gf.LevelSet(torch, **gf.LEVELSET_FULL, device=dev)
    dims = gf.LEVELSET_FULL["shape_xyz"]
    img, enc_s = encode_on_gpu(torch, lv.slab, dims, True)
    a = vbt.Asset(data=img, device=local_rank)
    a.build_page_table()
    rows = a.leaf_table()
    modes = np.bincount(rows[:, 1] & 3, minlength=4)
    out["config4_levelset"] = {"dims": list(dims) + [a.frames], "leaves": a.leaf_count,
                               "active_leaves": a.active_count, "grid4_leaves": int(modes[1]),
                               "mode2_leaves": int(modes[2]), "file_bytes": int(img.numel()), "encode_s": enc_s,
                               "full_frames": dense_timeline(torch, a, dev)}
    resident.append(a)
    names.append("config4_levelset")
    del img
    torch.cuda.empty_cache()
    # config 5: the serving mix over eight resident assets of the stated sizes -- the plume (config 2),
    # the fire's three fields (config 3), the level set (config 4), the scientific field 512^3 x 64
    # (config 5's own field, reference-encoded) and the two small scenes of configs 1 and 4
    more, more_names, skipped = open_assets(vbt, ["cfg2_plume", "cfg5_sci", "cfg1_blobs", "cfg4_sdf_small"],
                                            local_rank)
    if not args.no_serve:
        out["config5_serving"] = run_serving(args, local_rank, resident + more, names + more_names)
        out["config5_serving"]["assets_skipped"] = skipped
        out["config5_serving"]["resident_file_bytes"] = int(sum(x.info.payload_words * 4 for x in resident + more))
    for x in resident + more:
        x.close()
    out["note"] = ("fields generated and encoded on the GPU from their seeds; timings are device time with "
                   "the asset resident; encode_s is wall time of generation + encode + copy to host")
    return out


# ------------------------------------------------------------------------------ writer
def run_writer(args, local_rank, reps=5):
    """The VBTPACK4 writer on one B200 (vbt_pack_leaves: every leaf's control streams packed and the
    leaves assembled into the payload, one call) for the plume (32,768 leaves) and the config-4
    style level set (Mode2 shell leaves), stream arrays resident; device time of the call, its
    one host round trip for the payload size included.  Beside it the reference's own packer
    (packRenderTemporalControlStream + buildRenderTemporalPackedLeafBytes + the payload
    concatenation, oracle/_ref) on all host threads over the same arrays; both outputs are
    checked against the file."""
    import torch
    import vbt_b200 as vbt
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from leafstreams import streams_from_file
    dev = f"cuda:{local_rank}"
    out = {}
    for name in ("cfg2_plume", "mix_sdf"):
        path = os.path.join(ROOT, "assets", name + ".vbtp")
        if not os.path.exists(path):
            continue
        leaves, arr, _ = streams_from_file(path)
        raw = open(path, "rb").read()
        h = np.frombuffer(raw[8:52], np.uint32)
        off_at = 52 + 4 * int(h[10])
        want = np.frombuffer(raw[off_at + 4 * (int(h[8]) + 1):], np.uint32)
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a).view(dt)).to(dev) if a.size else None  # noqa: E731
        d_leaves = torch.from_numpy(leaves.view(np.uint8).copy()).to(dev)
        d = [t(arr["descriptors"], np.int32), t(arr["bins"], np.uint8), t(arr["key_frames"], np.int16),
             t(arr["key_values"], np.float32), t(arr["occupancy"], np.uint8)]
        n = leaves.shape[0]
        d_off = torch.empty(n + 1, dtype=torch.int32, device=dev)
        d_pay = torch.empty(want.size + 64, dtype=torch.int32, device=dev)
        s = torch.cuda.Stream(device=dev)
        s.wait_stream(torch.cuda.current_stream(dev))
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        with torch.cuda.stream(s):
            vbt.pack_leaves(d_leaves, *d, d_off, d_pay, stream=s)
            for e0, e1 in ev:
                e0.record(s)
                total = vbt.pack_leaves(d_leaves, *d, d_off, d_pay, stream=s)
                e1.record(s)
        s.synchronize()
        ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)
        ok = total == want.size and np.array_equal(d_pay[:total].cpu().numpy().view(np.uint32), want)
        entry = {"leaves": n, "active_leaves": int(((leaves["header"] & 3) != 0).sum()),
                 "mode2_leaves": int(((leaves["header"] & 3) == 2).sum()), "payload_bytes": int(total) * 4,
                 "call_ms": ms, "leaves_per_s": n / (ms * 1e-3), "payload_gb_per_s": total * 4 / (ms * 1e-3) / 1e9,
                 "equals_file": bool(ok), "gpu_launches_per_call": 3}
        if not args.no_cpu:
            try:
                from oracle.oracle import Reference
                ref = Reference()
                ref.pack_leaves(leaves, arr)
                t0 = time.perf_counter()
                for _ in range(3):
                    r_off, r_pay = ref.pack_leaves(leaves, arr, threads=os.cpu_count())
                el = (time.perf_counter() - t0) / 3
                entry["cpu_reference"] = {"ms": el * 1e3, "leaves_per_s": n / el, "cores": os.cpu_count(),
                                          "kind": "reference", "equals_file": bool(np.array_equal(r_pay, want))}
                entry["speedup_vs_cpu_reference"] = el * 1e3 / ms
            except (OSError, FileNotFoundError):
                pass
        out[name] = entry
    return out or {"skipped": "assets not generated"}


# ------------------------------------------------------------------------------ arms
def run_reference(args, rank, world):
    """The reference's own CPU decoder on the host cores, same metric and workload; each step is
    a bounded sample of the 96-frame timeline (the frames that fit in about 3 s)."""
    if rank != 0:
        return 0
    cpu = CpuDecoder(args.asset)
    per_frame_s = cpu.n_active * 512 / cpu.rate(1.0)[0]
    fps = max(1, min(cpu.frames, int(3.0 / max(per_frame_s, 1e-9))))
    times, t_next = [], 0
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for _ in range(fps):
            cpu.frame(t_next % cpu.frames)
            t_next += 1
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    value = cpu.n_active * 512 * fps * len(times) / sum(times)
    sample = f"{fps} of {cpu.frames} frames per step ({cpu.n_active} active leaves), {cpu.cores} threads"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "asset": os.path.basename(args.asset), "active_leaves": cpu.n_active,
                       "frames_per_step": fps},
            "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": cpu.cores, "kind": cpu.kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, local_rank, world):
    import torch
    import vbt_b200 as vbt

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    stream = torch.cuda.Stream(device=dev)
    a = vbt.Asset(args.asset, device=local_rank)
    T, n_active = a.frames, a.active_count
    frames = list(range(T))
    stride = n_active * 512
    cache = torch.empty((T, max(n_active, 1), 512), dtype=torch.float32, device=dev)
    # launch shape chosen by the library's autotuner on this asset and output
    tuning = a.autotune(T, cache, stream=stream)
    stream.synchronize()
    fpl = tuning.frames_per_launch if tuning.variant == 0 else CHUNK
    chunks = [frames[i:i + fpl] for i in range(0, T, fpl)]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    rows = a.leaf_table()
    bytes_per_frame, n_act2 = algorithmic_bytes_per_frame(rows)
    assert n_act2 == n_active

    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2 + len(chunks))] for _ in range(args.steps)]

    def step(evs=None):
        with torch.cuda.stream(stream):
            if evs:
                evs[0].record(stream)
            a.build_page_table(stream)
            if evs:
                evs[1].record(stream)
            for i, ch in enumerate(chunks):
                a.decode_cache(ch, cache[ch[0]], frame_stride=stride, stream=stream)
                if evs:
                    evs[2 + i].record(stream)

    for _ in range(args.warmup):
        step()
    stream.synchronize()
    a.sync_status(stream)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
    t_begin = time.time()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        step(ev[k])
    stream.synchronize()
    torch.cuda.synchronize()
    t_end = time.time()
    if pg:
        pg.barrier()
    clocks = sampler.stop(t_begin, t_end) if sampler else None
    a.sync_status(stream)
    step_ms = [e[0].elapsed_time(e[-1]) for e in ev]
    pt_ms = [e[0].elapsed_time(e[1]) for e in ev]
    dec_ms = [e[1 + i].elapsed_time(e[2 + i]) for e in ev for i in range(len(chunks))]
    total_ms = float(sum(step_ms))
    total_ms = max_over_ranks(total_ms, pg, dev)
    voxels_per_step = n_active * 512 * T
    value = world * voxels_per_step * args.steps / (total_ms * 1e-3)

    # roofline of the dominant kernel (decode_kernel<cache>), per launch
    peak, peak_src = measured_peak()
    mean_launch_s = statistics.mean(dec_ms) * 1e-3
    alg_per_launch = [bytes_per_frame * len(ch) for ch in chunks]
    achieved = statistics.mean(alg_per_launch) / mean_launch_s / 1e9
    traffic = ncu_traffic(len(chunks[0])) if len({len(ch) for ch in chunks}) == 1 else None

    # the same step replayed from a captured CUDA graph (page table + all decode launches, one
    # cudaGraphLaunch), timed the same way
    a.decode_cache_timeline(0, T, cache, frame_stride=stride, graph=True, stream=stream)
    gev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()
            gev[k][0].record(stream)
            a.decode_cache_timeline(0, T, cache, frame_stride=stride, graph=True, stream=stream)
            gev[k][1].record(stream)
    stream.synchronize()
    a.sync_status(stream)
    graph_ms = max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in gev), pg, dev) / args.steps

    # plain path: per frame, page table + one-CTA-per-leaf launch (no batching, no persistence)
    plain_ms = None
    plain_out = torch.empty((max(n_active, 1), 512), dtype=torch.float32, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        for rep in range(2):
            flush.zero_()
            e0.record(stream)
            for t in frames:
                a.build_page_table(stream)
                a.decode_cache_plain(t, plain_out, stream)
            e1.record(stream)
    stream.synchronize()
    plain_ms = e0.elapsed_time(e1)
    a.sync_status(stream)
    plain_value = voxels_per_step / (plain_ms * 1e-3)

    # end-to-end through the C-ABI with host buffers: every step re-uploads the file image from
    # pinned host memory (vbt_asset_upload: copies, walk, key order), builds the page table,
    # decodes the timeline and copies the whole cache back to pinned host memory.  Steps are
    # pipelined over three streams -- upload k+1 once decode k is done, decode k+1 into the other
    # of two cache buffers, the device-to-host copy of k meanwhile -- so the PCIe copies of
    # consecutive steps overlap each other and the decode, as a serving loop would run them.
    e2e = None
    if not args.no_e2e:
        image = np.fromfile(args.asset, dtype=np.uint8)
        h_img = torch.from_numpy(image).pin_memory()
        h_out = [torch.empty((T, max(n_active, 1), 512), dtype=torch.float32).pin_memory() for _ in range(2)]
        caches = [cache, torch.empty_like(cache)]
        s_in, s_dec, s_out = torch.cuda.Stream(device=dev), stream, torch.cuda.Stream(device=dev)
        e2e_steps = max(3, min(args.steps, 8))
        nsteps = 2 + e2e_steps
        up = [torch.cuda.Event() for _ in range(nsteps)]
        dec = [torch.cuda.Event() for _ in range(nsteps)]
        out_done = [torch.cuda.Event() for _ in range(nsteps)]
        ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for k in range(nsteps):
            if k == 2:
                s_in.wait_event(out_done[1])   # the warm-up steps are finished
                ee0.record(s_in)
            if k > 0:
                s_in.wait_event(dec[k - 1])
            a.upload(h_img, s_in)
            up[k].record(s_in)
            s_dec.wait_event(up[k])
            if k > 1:
                s_dec.wait_event(out_done[k - 2])   # its cache buffer has been copied out
            buf = caches[k % 2]
            with torch.cuda.stream(s_dec):
                a.build_page_table(s_dec)
                for ch in chunks:
                    a.decode_cache(ch, buf[ch[0]], frame_stride=stride, stream=s_dec)
            dec[k].record(s_dec)
            s_out.wait_event(dec[k])
            with torch.cuda.stream(s_out):
                h_out[k % 2].copy_(buf, non_blocking=True)
            out_done[k].record(s_out)
        ee1.record(s_out)
        torch.cuda.synchronize(dev)
        a.sync_status(s_dec)
        e2e_ms = ee0.elapsed_time(ee1) / e2e_steps
        e2e_ms = max_over_ranks(e2e_ms, pg, dev)
        e2e = {"value": world * voxels_per_step / (e2e_ms * 1e-3), "unit": "voxels/s",
               "h2d_bytes_per_step": int(image.nbytes), "d2h_bytes_per_step": int(cache.numel() * 4),
               "ms_per_step": e2e_ms, "pipelined": "upload, decode and copy-back of consecutive steps overlap"}
        del caches[1]

    full_frame = None
    if rank == 0 and world == 1 and not args.no_full_frame:
        full_frame = run_full_frame(args, local_rank, a, rows)

    sampler = None
    if rank == 0 and world == 1 and not args.no_sampler:
        sampler = run_sampler(args, local_rank)

    keyframes = None
    if rank == 0 and world == 1 and not args.no_keyframes:
        keyframes = run_keyframes(args, local_rank)

    writer = None
    if rank == 0 and world == 1 and not args.no_writer:
        writer = run_writer(args, local_rank)

    ref_queries = None
    if rank == 0 and world == 1 and not args.no_ref_queries:
        ref_queries = run_reference_queries(args, local_rank)

    window = window_render = None
    if rank == 0 and world == 1 and not args.no_window:
        window = run_window(args, local_rank)
        window_render = run_window_render(args, local_rank)

    full_size = None
    if rank == 0 and world == 1 and args.full_size:
        full_size = run_full_size(args, local_rank)

    serving = None
    if rank == 0 and world == 1 and not args.no_serve:
        serving = run_serving(args, local_rank)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        dec = CpuDecoder(args.asset)
        v, sample = dec.rate(args.cpu_seconds)
        cpu = {"value": v, "unit": "voxels/s", "cores": dec.cores, "kind": dec.kind, "sample": sample}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "asset": os.path.basename(args.asset), "leaves": a.leaf_count,
                           "active_leaves": n_active, "frames_per_step": T, "frames_per_launch": fpl,
                           "l2": "flushed before every timed step (256 MiB write)",
                           "cache_ring_bytes": int(cache.numel() * 4), "parallelism": f"replicas x{world}"},
                "roofline": {"bound": "hbm", "kernel": "decode_leaf_kernel<cache>", "achieved": achieved, "peak": peak,
                             "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                             "traffic_source": "profiles/decode_leaf_cfg2.md: dram bytes of one ncu capture of "
                                               "this kernel on this workload (not measured by this run)"
                             if traffic is not None else None,
                             "algorithmic_bytes_per_launch": int(statistics.mean(alg_per_launch)),
                             "launch_ms": statistics.mean(dec_ms), "peak_source": peak_src},
                "kernels_ms": {"page_table": statistics.mean(pt_ms), "decode_per_launch": statistics.mean(dec_ms)},
                "graph": {"value": world * voxels_per_step / (graph_ms * 1e-3), "unit": "voxels/s",
                          "ms_per_step": graph_ms, "launches_per_step": 1},
                "tuning": {"variant": ["leaf per CTA", "leaf per warp"][tuning.variant],
                           "frames_per_launch": tuning.frames_per_launch, "grid": tuning.grid,
                           "ms_per_frame": tuning.ms_per_frame, "ms_per_frame_untuned": tuning.ms_per_frame_default},
                "plain": {"value": plain_value, "unit": "voxels/s", "ms_per_step": plain_ms,
                          "launches_per_step": 2 * T, "speedup_batched_vs_plain": value / world / plain_value},
                "cpu_baseline": cpu, "e2e": e2e, "serving": serving, "precision_window": window,
                "precision_window_render": window_render, "full_frame": full_frame, "ray_sampler": sampler,
                "keyframe_pass": keyframes, "writer": writer, "full_size": full_size, "point_queries_vs_reference_cuda": ref_queries,
                "gpu_launches": args.steps * (1 + len(chunks)),
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    a.close()
    if pg:
        pg.destroy_process_group()
    return 0


def main():
    args = parse()
    rank, local_rank, world = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, local_rank, world)


if __name__ == "__main__":
    sys.exit(main())
