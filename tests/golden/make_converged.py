"""Writes the converged-image fixtures: 16384-spp renders of fixed crop windows by the reference
engine's own CPU path (shipping build, oracle/_ref/libphoton_ref_fast.so), one file per workload.

    python tests/golden/make_converged.py [cornell|knot|media|room ...] [--spp 16384] [--threads N]

Each workload is built at the size its configuration states and rendered through the seeded
tracePixel loop over the windows in CONFIGS (x0, y0, w, h in frame pixels), samples
[0, spp) of the workload's Sobol seed.  The GPU test (tests/test_gpu_converged.py) renders the
same windows and samples with the device and holds relMSE (mean over pixels and channels of
(x − ref)² / (ref² + 0.01)) at most 1e-3.  Rendering is chunked (2048 samples a chunk) and
resumable: partial sums are kept in --work (default: a folder in the system temp dir).
Output: converged_<name>.npz with `mean` (windows, h, w, 3) float32, `count` (windows, h, w)
uint32, `rects`, `spp`, `seed`.
"""
from __future__ import annotations

import argparse
import os
import pathlib
import sys
import tempfile
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def _scenes():
    sys.path.insert(0, str(ROOT))
    import pe_pkg
    pe_pkg.load()
    import importlib
    return importlib.import_module("photon_engine_b200.scenes")


def build(name: str):
    """(scene, camera, settings) of a workload at its configured size."""
    S = _scenes()
    if name == "cornell":   # 36 triangles, 256², depth 8, RR after 3, Sobol seed 0
        return S.cornell_box(256, 256, 64, 8, seed=0)
    if name == "knot":      # ~1M triangles, 2048×1024 sky + softbox, 1920×1080, depth 12
        return S.torus_knot_scene(1920, 1080, 256, 12)
    if name == "media":     # 2000 LED triangles, glass, volumes, SSS slab, ~200k triangles, 1280×720, depth 24
        return S.media_scene(1280, 720, 512, 24)
    if name == "room":      # ~0.5M-triangle room lit through a 1×1 m window, 1920×1080, depth 12
        return S.room_scene(1920, 1080, 64, 12)
    raise KeyError(name)


# Crop windows (x0, y0, w, h) in frame pixels: the whole Cornell frame; on the others four 128²
# windows over highlights, shadows, media and emitters.
CONFIGS = {
    "cornell": [(0, 0, 256, 256)],
    "knot": [(680, 340, 128, 128),     # cyan clearcoat tube, sun highlight
             (1380, 700, 128, 128),    # ground shadow of the knot
             (200, 100, 128, 128),     # sky gradient over the horizon
             (1000, 660, 128, 128)],   # metallic tube in front
    "media": [(200, 40, 128, 128),     # LED strip (2000 emissive triangles)
              (316, 288, 128, 128),    # left sphere
              (824, 276, 128, 128),    # right sphere
              (576, 300, 128, 128)],   # subsurface slab over the absorbing liquid
    "room": [(916, 576, 128, 128),     # sun patch on the floor
             (1136, 416, 128, 128),    # metallic knot in indirect light
             (696, 336, 128, 128),     # knot in shadow
             (256, 96, 128, 128)],     # ceiling corner, indirect only
}


def generate(name: str, spp: int, threads: int, work: pathlib.Path, chunk: int = 2048) -> pathlib.Path:
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    scene, cam, st = build(name)
    scene.build_accelerator()  # also checks the scene builds on the product side
    ref = oracle.RefScene(scene, fast=True)
    rects = CONFIGS[name]
    work.mkdir(parents=True, exist_ok=True)
    out_mean, out_count = [], []
    for k, rect in enumerate(rects):
        x0, y0, w, h = rect
        part = work / f"{name}_{k}_{spp}.npz"
        acc = np.zeros((h, w, 3), np.float64)
        cnt = np.zeros((h, w), np.uint64)
        done = 0
        if part.exists():
            z = np.load(part)
            acc, cnt, done = z["acc"], z["cnt"].astype(np.uint64), int(z["done"])
        while done < spp:
            n = min(chunk, spp - done)
            t0 = time.perf_counter()
            mean, c = ref.render_rect(cam, st, rect, done, n, threads)
            acc += mean.astype(np.float64) * c[..., None]
            cnt += c
            done += n
            np.savez(part, acc=acc, cnt=cnt, done=done)
            print(f"{name} window {k}: {done}/{spp} spp ({time.perf_counter() - t0:.1f} s a chunk)", flush=True)
        out_mean.append((acc / np.maximum(cnt, 1)[..., None]).astype(np.float32))
        out_count.append(cnt.astype(np.uint32))
    path = HERE / f"converged_{name}.npz"
    np.savez_compressed(path, mean=np.stack(out_mean), count=np.stack(out_count), rects=np.array(rects, np.int32),
                        spp=np.int32(spp), seed=np.uint64(st.seed))
    return path


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*", default=list(CONFIGS))
    ap.add_argument("--spp", type=int, default=16384)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--work", default=os.path.join(tempfile.gettempdir(), "photon_converged"))
    args = ap.parse_args()
    for name in args.names:
        print(generate(name, args.spp, args.threads, pathlib.Path(args.work)))


if __name__ == "__main__":
    main()
