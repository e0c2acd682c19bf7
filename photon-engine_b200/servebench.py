"""Served-mix benchmark: a Poisson stream of render requests over four resident scenes, run once
through the request server (continuous batching, HBM-budget admission, least-work-first) and
once through the plain one-request-at-a-time loop of the drop-in API (set the request's scene,
render it into a host film).  Both see the same arrival times.

Mix: scenes {Cornell box, 1M-triangle torus knot, many-light/media scene, 5.2M-triangle grid};
resolution from {256², 512², 1280×720, 1920×1080} and spp from {16, 64, 256, 1024}, uniform;
arrivals Poisson at ``rate`` requests/s.  Preview probes (512², 16 spp) arrive through the same
window at ``probe_rate``/s: their latency is the served path's interactive figure.

Latency of a request = film in host memory − arrival (the served path's take() included).
Aggregate throughput = Σ paths of the requests / (last completion − first arrival).
"""
from __future__ import annotations

import threading
import time

import numpy as np

RESOLUTIONS = [(256, 256), (512, 512), (1280, 720), (1920, 1080)]
SPPS = [16, 64, 256, 1024]
DEPTHS = {"cornell": 8, "knot": 12, "media": 24, "grid": 12}


def build_scenes(pe, quick: bool = False):
    from . import scenes as S
    out = {}
    c, _, _ = S.cornell_box()
    out["cornell"] = c
    if quick:
        k, _, _ = S.torus_knot_scene(nu=512, nv=32, env_size=(256, 128))
        m, _, _ = S.media_scene(n_leds=200, sphere_res=(48, 24), cyl_res=(32, 6), slab_res=4)
        g, _, _ = S.instanced_grid_scene(nx=2, nz=2, nu=256, nv=32, env_size=(256, 128))
    else:
        k, _, _ = S.torus_knot_scene()
        m, _, _ = S.media_scene()
        g, _, _ = S.instanced_grid_scene()
    out["knot"], out["media"], out["grid"] = k, m, g
    for sc in out.values():
        sc.build_accelerator()
    return out


def make_stream(n: int, rate: float, probes: int, probe_rate: float, seed: int = 2024):
    """[(arrival_s, scene, w, h, spp, is_probe)] sorted by arrival."""
    rng = np.random.default_rng(seed)
    names = ["cornell", "knot", "media", "grid"]
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    reqs = []
    for i in range(n):
        w, h = RESOLUTIONS[int(rng.integers(0, 4))]
        reqs.append((float(t[i]), names[int(rng.integers(0, 4))], w, h, SPPS[int(rng.integers(0, 4))], False))
    tp = np.cumsum(rng.exponential(1.0 / probe_rate, probes))
    for i in range(probes):
        reqs.append((float(tp[i]), names[int(rng.integers(0, 4))], 512, 512, 16, True))
    return sorted(reqs, key=lambda r: r[0])


def _settings(pe, name, w, h, seed):
    return pe.RenderSettings(width=w, height=h, max_bounces=DEPTHS[name], seed=seed)


def run_plain(pe, device, scenes, stream):
    from . import scenes as S
    t0 = time.perf_counter()
    current = None
    lat, done_at, paths = [], [], 0
    for i, (arr, name, w, h, spp, probe) in enumerate(stream):
        now = time.perf_counter() - t0
        if now < arr:
            time.sleep(arr - now)
        if current != name:
            device.set_scene(scenes[name])
            current = name
        film = pe.Film(w, h)
        device.render(S.camera_for(name, w, h), _settings(pe, name, w, h, i), pe.RenderTargets(beauty=film), 0, spp)
        t = time.perf_counter() - t0
        lat.append((t - arr, probe))
        done_at.append(t)
        paths += w * h * spp
    return lat, max(done_at) - stream[0][0], paths


def run_served(pe, device, scenes, stream, budget_bytes):
    from . import scenes as S
    lat = [None] * len(stream)
    done_at = [0.0] * len(stream)
    with pe.RenderServer(device, budget_bytes) as srv:
        sid = {name: srv.add_scene(sc) for name, sc in scenes.items()}
        t0 = time.perf_counter()
        ids = [None] * len(stream)
        ready = [threading.Event() for _ in stream]

        def collect(i):
            ready[i].wait()
            srv.wait(ids[i])
            srv.take(ids[i])
            t = time.perf_counter() - t0
            lat[i] = (t - stream[i][0], stream[i][5])
            done_at[i] = t

        threads = [threading.Thread(target=collect, args=(i,)) for i in range(len(stream))]
        for th in threads:
            th.start()
        for i, (arr, name, w, h, spp, probe) in enumerate(stream):
            now = time.perf_counter() - t0
            if now < arr:
                time.sleep(arr - now)
            ids[i] = srv.submit(sid[name], S.camera_for(name, w, h), _settings(pe, name, w, h, i), spp)
            ready[i].set()
        for th in threads:
            th.join()
        stats = srv.stats()
    paths = sum(w * h * spp for (_, _, w, h, spp, _) in stream)
    return lat, max(done_at) - stream[0][0], paths, stats


def _pct(xs, q):
    return float(np.percentile(np.asarray(xs) * 1000.0, q)) if xs else None


def summarize(lat, span_s, paths):
    allv = [l for l, _ in lat]
    probes = [l for l, p in lat if p]
    return {"paths_per_s": paths / span_s, "span_s": span_s, "requests": len(lat),
            "p50_ms": _pct(allv, 50), "p99_ms": _pct(allv, 99),
            "preview_p50_ms": _pct(probes, 50), "preview_p99_ms": _pct(probes, 99), "previews": len(probes)}


def run(pe, device, n_requests=24, rate=40.0, probes=24, probe_rate=8.0, budget_bytes=32 << 30, quick=False):
    from . import scenes as S
    scenes = build_scenes(pe, quick)
    stream = make_stream(n_requests, rate, probes, probe_rate)
    # warm both paths (first uploads, kernel loads) on a small request per scene
    for name, sc in scenes.items():
        device.set_scene(sc)
        device.render(S.camera_for(name, 64, 64), _settings(pe, name, 64, 64, 0), pe.RenderTargets(beauty=pe.Film(64, 64)),
                      0, 1)
    lat_s, span_s, paths_s, stats = run_served(pe, device, scenes, stream, budget_bytes)
    lat_p, span_p, paths_p = run_plain(pe, device, scenes, stream)
    served = summarize(lat_s, span_s, paths_s)
    plain = summarize(lat_p, span_p, paths_p)
    served.update({"waves": int(stats.waves), "segments": int(stats.segments), "film_bytes_peak": int(stats.film_bytes_peak),
                   "device_busy_s": stats.busy_ms / 1000.0})
    return {"served": served, "plain": plain, "speedup": served["paths_per_s"] / plain["paths_per_s"],
            "mix": {"requests": n_requests, "rate_per_s": rate, "probes": probes, "probe_rate_per_s": probe_rate,
                    "resolutions": RESOLUTIONS, "spp": SPPS, "scenes": list(scenes),
                    "triangles": {k: int(v.info.triangles) for k, v in scenes.items()}}}
