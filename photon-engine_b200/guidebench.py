"""Time to a relMSE target, plain against guided sampling, on the indirect-lit room (a closed
10 × 8 × 3 m interior lit through one 1 × 1 m window by the sky, three torus knots, a sphere, two
tables).

Both sides render through the drop-in API (``CudaDevice.render`` into a host film) from sample 0,
and the clock is the wall time of those calls, so the guided side pays for its inference, its
training (one Adam step per wave) and its smaller waves.  relMSE = mean((x − r)² / (r² + 0.01))
(the reference's compare script) against a converged plain render of a disjoint sample range,
on images scaled so that the converged mean is 0.18 (the room is dark at its raw exposure, and
the + 0.01 term would hide all error there).  Each curve is averaged over independent Sobol
seeds.  The target is the relMSE the plain renderer reaches at ``target_spp``; the result is the
ratio of the plain and guided times to reach it.  The reference's SD-tree guiding runs beside
them the same way.
"""
from __future__ import annotations

import time

import numpy as np


def _curve(pe, dev, cam, st, ref, k, spp, batch, seeds, guided, warmup=16, lr=3e-3):
    """(seconds, spp, relMSE) after each render call; `guided`: 0 plain, 1 the learned
    proposal (a fresh network, trained online), 2 the SD-tree (trained over samples 0-31)."""
    lib = pe._capi.load()
    curves = []
    for seed in seeds:
        st.seed = seed
        if guided == 1:
            # a fresh network for every run: its training is part of the time
            pe._capi.check(lib.pe_device_guide_reset(dev.handle, int(seed), None, None))
            pe._capi.check(lib.pe_device_set_guiding(dev.handle, 1, warmup, lr))
        elif guided == 2:
            pe._capi.check(lib.pe_device_set_guiding(dev.handle, 2, 0, 0.0))
        film = pe.Film(st.width, st.height)
        t, pts = 0.0, []
        for s0 in range(0, spp, batch):
            t0 = time.perf_counter()
            dev.render(cam, st, pe.RenderTargets(beauty=film), s0, batch)
            t += time.perf_counter() - t0
            img = film.resolve()
            pts.append((t, s0 + batch, pe.rel_mse(img * k, ref * k)))
        if guided:
            pe._capi.check(lib.pe_device_set_guiding(dev.handle, 0, 0, 0.0))
        curves.append(pts)
    # average over seeds at equal batch index
    n = min(len(c) for c in curves)
    return [(float(np.mean([c[i][0] for c in curves])), curves[0][i][1], float(np.mean([c[i][2] for c in curves])))
            for i in range(n)]


def _time_to(curve, target):
    """Time at which the curve first reaches `target` (linear in log relMSE between points)."""
    prev = None
    for t, _, e in curve:
        if e <= target:
            if prev is None:
                return t
            t0, e0 = prev
            a = (np.log(e0) - np.log(target)) / max(1e-12, np.log(e0) - np.log(e))
            return t0 + a * (t - t0)
        prev = (t, e)
    return None


def run(pe, dev, width=320, height=180, ref_spp=8192, spp=1024, target_spp=256, seeds=(11, 22)):
    from . import scenes
    scene, cam, st = scenes.room_scene(width, height, 32, 8, knot_res=(256, 32), env_size=(512, 256))
    scene.build_accelerator()
    dev.set_scene(scene)
    lib = pe._capi.load()
    pe._capi.check(lib.pe_device_set_guiding(dev.handle, 0, 0, 0.0))
    # converged image: plain, a disjoint sample range
    ref_film = pe.Film(width, height)
    for s0 in range(1 << 22, (1 << 22) + ref_spp, 1024):
        dev.render(cam, st, pe.RenderTargets(beauty=ref_film), s0, 1024)
    ref = ref_film.resolve()
    k = 0.18 / float(ref.mean())
    # warm both paths once (kernel loads, first allocations)
    dev.render(cam, st, pe.RenderTargets(beauty=pe.Film(width, height)), 1 << 23, 4)
    plain = _curve(pe, dev, cam, st, ref, k, spp, 16, seeds, guided=0)
    guided = _curve(pe, dev, cam, st, ref, k, spp, 4, seeds, guided=1)
    sdtree = _curve(pe, dev, cam, st, ref, k, spp, 16, seeds, guided=2)
    target = next(e for t, s, e in plain if s >= target_spp)
    tp, tg, ts = _time_to(plain, target), _time_to(guided, target), _time_to(sdtree, target)
    at = lambda c, s: next(e for t, n, e in c if n >= s)
    return {"target_relmse": target, "target_spp": target_spp, "plain_s": tp, "guided_s": tg, "sdtree_s": ts,
            "time_to_relmse_speedup": (tp / tg) if (tp and tg) else None,
            "sdtree_time_to_relmse_speedup": (tp / ts) if (tp and ts) else None,
            "equal_spp_relmse": {str(s): {"plain": at(plain, s), "guided": at(guided, s), "sdtree": at(sdtree, s)}
                                 for s in (64, 256, spp)},
            "plain_ms_per_spp": 1000.0 * plain[-1][0] / plain[-1][1],
            "guided_ms_per_spp": 1000.0 * guided[-1][0] / guided[-1][1],
            "sdtree_ms_per_spp": 1000.0 * sdtree[-1][0] / sdtree[-1][1],
            "config": {"scene": "indirect-lit room (window 1x1 m)", "width": width, "height": height, "max_depth": 8,
                       "reference_spp": ref_spp, "spp": spp, "seeds": list(seeds),
                       "plain_batch_spp": 16, "guided_batch_spp": 4}}
