#!/usr/bin/env python3
"""Generate tests/golden/keyframes.npz from the reference encoder's own keyframe detector.

Runs in the development container only: it needs oracle/_ref/libkfref.so, which oracle/Makefile
builds from the reference sources (detectDensityKeyFrames and reconstructFromKeys,
src/render_temporal_kf_probe_main.cpp:2080-2201).  Seeded series of several shapes -- a Gaussian
pulse over noise, constants, near-constants under the epsilon floor, values dithering around the
render cutoff, random walks, sparse spikes, sinusoids, all-zero -- with frame counts from 1 to 200,
under four profiles (the encoder's defaults; level-set iso protection with the cutoff off; no
gamma and no cutoff protection; iso protection and cutoff protection together).  Recorded per
case: the series, the profile index, the reference's keys, its usedCutoffProtect flag and its
reconstruction.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import KeyframeReference, VoKeyframeProfile  # noqa: E402

PROFILES = [dict(), dict(iso_surface_protect=1, iso_band=0.1, render_cutoff=-1.0),
            dict(gamma_delta=0.0, eps_rel=0.05, cutoff_temporal_protect=0),
            dict(iso_surface_protect=1, iso_band=0.05, iso_value=0.2)]
FRAMES = [1, 2, 3, 5, 24, 33, 64, 96, 120, 200]
KINDS = 8


def series(rng, kind, T):
    t = np.arange(T)
    if kind == 0:
        c, w = rng.uniform(0, T), rng.uniform(2, 10)
        return rng.normal(0, 0.01, T) + 0.5 * np.exp(-((t - c) / w) ** 2)
    if kind == 1:
        return np.full(T, rng.uniform(0, 1))
    if kind == 2:
        return np.full(T, 0.3) + rng.normal(0, 1e-7, T)
    if kind == 3:
        return rng.uniform(0, 0.0006, T)
    if kind == 4:
        return rng.normal(0, 1, T).cumsum() * 0.1
    if kind == 5:
        return np.where(rng.random(T) < 0.5, 0.0, rng.uniform(0, 1, T))
    if kind == 6:
        return np.sin(t * rng.uniform(0.01, 0.5)) * rng.uniform(0.1, 5)
    return np.zeros(T)


def main():
    ref = KeyframeReference()
    rng = np.random.default_rng(20240611)
    vals, keys, recon = [], [], []
    meta = []          # (frames, kind, profile, value offset, key offset, key count, used)
    voff = koff = 0
    for T in FRAMES:
        for kind in range(KINDS):
            for pi, pk in enumerate(PROFILES):
                for _ in range(3):
                    v = series(rng, kind, T).astype(np.float32)
                    prof = VoKeyframeProfile(**pk)
                    k, used = ref.detect_keyframes(v, prof)
                    r = ref.reconstruct(v, k)
                    meta.append((T, kind, pi, voff, koff, len(k), int(used)))
                    vals.append(v)
                    keys.append(k.astype(np.int32))
                    recon.append(r)
                    voff += T
                    koff += len(k)
    np.savez_compressed(os.path.join(HERE, "keyframes.npz"), meta=np.array(meta, np.int64),
                        values=np.concatenate(vals), keys=np.concatenate(keys), recon=np.concatenate(recon),
                        profiles=np.array([repr(p) for p in PROFILES]))
    print(len(meta), "cases")


if __name__ == "__main__":
    main()
