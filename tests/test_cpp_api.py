"""The C++ decoder API (include/vbt/*.h, implemented in vbt_b200/csrc/facade.cpp) through C++
test programs under tests/cpp/ that restate the reference's own C++ tests.

host_api_test needs no GPU: payload/reader/stream format functions against the reference's test
cases and the C oracle, plus query generation, DCT helpers, stream packing and leaf parsing
against golden fixtures that the reference produced (tests/golden/make_golden.py).
decode_api_test needs a GPU: every decode call against the oracle, bit for bit.
"""
import json
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden_asset

CPP = os.path.join(ROOT, "tests", "cpp")
LIB_DIR = os.path.join(ROOT, "vbt_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")


def compile_program(name, out_dir, cuda_runtime=False):
    """g++ the test program against libvbt_b200.so and liboracle.so (both built by build()), and
    the CUDA runtime when the program calls it itself."""
    for lib in (os.path.join(LIB_DIR, "libvbt_b200.so"), os.path.join(ORACLE_DIR, "liboracle.so")):
        if not os.path.exists(lib):
            pytest.skip(f"{os.path.basename(lib)} not built (run __graft_entry__.build())")
    exe = os.path.join(out_dir, name)
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", ORACLE_DIR,
           "-I", CPP, os.path.join(CPP, name + ".cpp"), "-o", exe, "-L", LIB_DIR, "-lvbt_b200", "-L", ORACLE_DIR,
           "-loracle", f"-Wl,-rpath,{LIB_DIR}:{ORACLE_DIR}"]
    if cuda_runtime:
        cmd += ["-I", "/usr/local/cuda/include", "-L", "/usr/local/cuda/lib64", "-lcudart",
                "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.fixture(scope="module")
def host_run(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("cpp_host"))
    exe = compile_program("host_api_test", d)
    fx = np.load(os.path.join(GOLDEN, "host_api.npz"))
    streams = np.load(os.path.join(GOLDEN, "streams.npz"))
    payload = np.load(os.path.join(GOLDEN, "payload_cases.npz"))
    lines = []
    # stream constructions of streams.npz, in its generation order
    order = [(c, b, f, d_, h) for c in (0, 1) for b in (4, 8) for f in sorted(set(streams["meta"][:, 2].tolist()))
             for d_, h in ((1, -1), (0, -1), (0, 0), (0, 255))]
    for c, b, f, d_, h in order:
        # the generator's series: float32 sin(0.19 t) as numpy computes it
        series = np.sin(np.arange(f, dtype=np.float32) * np.float32(0.19)).astype(np.float32).view(np.uint32)
        lines.append(f"S {c} {b} {f} {d_} {h} " + " ".join(format(int(v), "x") for v in series))
    for row in fx["qmeta"]:
        lines.append("Q " + " ".join(str(int(v)) for v in row))
    soff = 0
    for n, keep, weighted, _ in fx["dmeta"]:
        s = fx["series"][soff:soff + n].view(np.uint32)
        w = fx["weights"][soff:soff + n].view(np.uint32)
        soff += n
        words = [format(int(v), "x") for v in s] + ([format(int(v), "x") for v in w] if weighted else [])
        lines.append(f"D {n} {keep} {weighted} " + " ".join(words))
    names = sorted(payload.files)
    for k in names:
        lines.append("P " + payload[k].tobytes().hex())
    case_file = os.path.join(d, "cases.txt")
    out_file = os.path.join(d, "out.bin")
    open(case_file, "w").write("\n".join(lines) + "\n")
    assets = [golden_asset(n) for n in ("tiny_density", "tiny_levelset", "sci_small")]
    r = subprocess.run([exe, os.path.join(d, "scratch"), case_file, out_file] + assets, capture_output=True,
                       text=True, timeout=300)
    words = np.fromfile(out_file, np.uint32) if os.path.exists(out_file) else np.zeros(0, np.uint32)
    return r, words, order, fx, streams, payload, names


def test_host_api_program_passes(host_run):
    r = host_run[0]
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr


def _reader(words):
    pos = [0]

    def take(n):
        v = words[pos[0]:pos[0] + n]
        assert v.size == n, "output ended early"
        pos[0] += n
        return v
    return take, pos


def test_host_api_outputs_match_reference_fixtures(host_run):
    r, words, order, fx, streams, payload, names = host_run
    assert r.returncode == 0, r.stderr
    take, pos = _reader(words)
    # 1. packRenderTemporalControlStream == the reference's packer on every streams.npz construction
    meta, blob = streams["meta"], streams["bytes"]
    index = {}
    for i, m in enumerate(meta):
        index.setdefault((int(m[0]), int(m[1]), int(m[2])), []).append(i)
    seen = {}
    for c, b, f, d_, h in order:
        n = int(take(1)[0])
        got = take((n + 3) // 4).view(np.uint8)[:n]
        k = (c, b, f)
        j = index[k][seen.get(k, 0)]
        seen[k] = seen.get(k, 0) + 1
        want = blob[int(meta[j][5]):int(meta[j][5]) + int(meta[j][4])]
        assert np.array_equal(got, want), ("packed stream differs", k, d_, h)
    # 2. generateQueries / fillLeafIndices / sortQueriesByLeaf
    qoff = 0
    for row in fx["qmeta"]:
        cnt = int(row[6])
        gen = take(cnt * 5).reshape(cnt, 5)
        srt = take(cnt * 5).reshape(cnt, 5)
        assert np.array_equal(gen, fx["qgen"][qoff:qoff + cnt]), ("generated queries differ", row)
        assert np.array_equal(srt, fx["qsorted"][qoff:qoff + cnt]), ("sorted queries differ", row)
        qoff += cnt
    # 3. dctEncodeKeep[Weighted] / dctDecodeAt, bit for bit
    coff = soff = 0
    for n, keep, weighted, k in fx["dmeta"]:
        kk = int(take(1)[0])
        assert kk == k
        c = take(kk)
        dec = take(int(n))
        assert np.array_equal(c, fx["coeffs"][coff:coff + k].view(np.uint32)), ("dct coefficients", n, keep, weighted)
        assert np.array_equal(dec, fx["decoded"][soff:soff + n].view(np.uint32)), ("dct decode", n, keep, weighted)
        coff += k
        soff += n
    # 4. parseRenderTemporalPackedLeaf verdicts of the reference's payload test cases
    verdicts = json.load(open(os.path.join(GOLDEN, "payload_cases.json")))
    for name in names:
        n = int(take(1)[0])
        msg = take((n + 3) // 4).view(np.uint8)[:n].tobytes().decode()
        view = take(16)
        want = verdicts[name]
        assert (msg or None) == want["error"], (name, msg, want["error"])
        if want["error"] is None:
            assert view.tolist() == want["view"], name
    assert pos[0] == words.size


@pytest.mark.gpu
def test_decode_api_program(tmp_path, cuda):
    exe = compile_program("decode_api_test", str(tmp_path))
    render = [golden_asset("tiny_density"), golden_asset("tiny_levelset")]
    for n in ("cfg1_blobs", "cfg4_sdf_small"):
        p = os.path.join(ROOT, "assets", n + ".vbtp")
        if os.path.exists(p):
            render.append(p)
    r = subprocess.run([exe] + render + ["--sci", golden_asset("sci_small")], capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_facade_copies_and_latency(tmp_path, cuda):
    """Device copies of VbtFile objects: bounded without releaseDeviceCopy, never stale after an
    in-place change or a reload into the same object; and the scalar calls' latency."""
    exe = compile_program("facade_test", str(tmp_path), cuda_runtime=True)
    r = subprocess.run([exe, golden_asset("tiny_density"), golden_asset("sci_small")], capture_output=True, text=True,
                       timeout=600)
    print(r.stdout)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr
    lat = {ln.split()[1]: float(ln.split()[2]) for ln in r.stdout.splitlines() if ln.startswith("LATENCY")}
    assert set(lat) == {"decodeRenderTemporalLeafControlValue", "decodeScientificValueAtCpu"}
