"""Throughput benchmark of the B200 path tracer on the product-scale torus-knot workload.

Workload (one ``step``): four samples per pixel of a 1920×1080 frame of the ~1M-triangle torus
knot with eight Disney materials, a 2048×1024 HDR sky (sun lobe 60 % of power) and a softbox,
max depth 12 — i.e. 8,294,400 camera paths per step, one wave through the 2M path slots (generate,
then per bounce closest hit, shade, any hit and the refill of freed slots with the wave's next
paths, then tail and film), a batch of the 256-spp frame.  Metric: paths/s (W·H·spp / render seconds, the reference's
msamplesPerSecond definition).

``value``   device-resident: inputs in HBM, K steps into the resident film, CUDA events on the
            library's stream, max over ranks.
``e2e``     the same K steps through the public RenderDevice::render call with host films:
            camera + settings in, the frame's film (sum, count, sum of squares) read back and
            merged on the host every step.
``roofline`` closest-hit traversal kernel: algorithmic bytes (4-wide BVH nodes visited × 128 B +
            triangles tested × 48 B + ray record 32 B + hit record 16 B + queue index 4 B per
            ray, counted on the device over one untimed step) ÷ its CUDA-event time, against
            the measured HBM copy bandwidth.
``cpu_baseline`` the reference engine's own CPU path (built with its shipping flags) on the same
            scene and camera, all host threads, a bounded number of full-frame samples.

``--impl reference`` times only that CPU implementation (Renderer::renderSamples) on the same
            workload and step, four full-frame samples per step, with no product library loaded.
``--gpus N`` (torchrun) runs N independent replicas, each rendering its own sample indices:
the path does not shard further and needs no collective.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WIDTH, HEIGHT, DEPTH = 1920, 1080, 12
SPP_PER_STEP = 4  # one step = 4 samples per pixel of the 1080p frame (one wave of 8.3M paths)
NODE_BYTES, TRI_BYTES, RAY_BYTES, HIT_BYTES, QUEUE_BYTES = 128, 48, 32, 16, 4  # 4-wide BVH node: 128 B
L2_NOTE = ("inputs larger than L2: 140 MB resident scene + 0.6-1.2 GB of path state for the 4-8M paths in flight "
           "(L2 126 MB)")


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = "pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, pci_bus_id: str):
        self.pci = pci_bus_id.lower()
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            bus = f[0].lower()
            if self.pci and not (bus.endswith(self.pci[-12:]) or self.pci.endswith(bus[-12:])):
                continue
            rows.append(f)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def replica_sample_base(rank: int, warmup: int, steps: int) -> int:
    """First sample index of a replica: the counting pass, warm-up and timed steps of each rank
    use disjoint sample ranges [base, base + SPP_PER_STEP·(1 + warmup + steps))."""
    return rank * (warmup + steps + 8) * SPP_PER_STEP


def step_samples(base: int, warmup: int, k: int) -> int:
    """First sample of timed step k after `warmup` warm-up steps (warm-up step w: step_samples(base, 0, w))."""
    return base + SPP_PER_STEP * (1 + warmup + k)


def max_over_ranks(value: float, pg, device: str) -> float:
    """Whole-job time: the maximum over ranks (all ranks call this in the same order)."""
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def _scenegen():
    """The workload generator (plain numpy), loaded by file path so that the reference arm
    imports no product module and loads no product library."""
    import importlib.util
    name = "_photon_scenegen"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, ROOT / "photon-engine_b200" / "scenegen.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def workload_description(width=WIDTH, height=HEIGHT, nu=4096, nv=128, env_size=(2048, 1024)):
    return _scenegen().torus_knot(width, height, 256, DEPTH, nu, nv, env_size)


def workload_config(desc) -> dict:
    """The config both arms report (one workload, one step definition)."""
    st = desc["settings"]
    return {"workload": "torus-knot 1M tris, 8 Disney materials, 2048x1024 HDR sky + softbox, 1920x1080, depth 12",
            "spp_per_step": SPP_PER_STEP, "paths_per_step": st["width"] * st["height"] * SPP_PER_STEP,
            "triangles": _scenegen().triangle_count(desc), "l2": L2_NOTE, "parallelism": "replicas x1"}


def build_workload(pe):
    import importlib
    sc = importlib.import_module("photon_engine_b200.scenes")
    desc = workload_description()
    scene, cam, st = sc.from_description(desc)
    scene.build_accelerator()
    return scene, cam, st, desc


def cpu_reference(desc, min_seconds: float, max_spp: int, first: int = 0):
    """The reference's stock CPU path (Renderer::renderSamples, shipping build) on all host
    threads: full-frame samples until min_seconds."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    ref = oracle.ref_scene_from_description(desc, fast=True)
    cam = oracle.DescCamera(desc["camera"], fast=True)
    st = oracle.DescSettings(desc["settings"])
    threads = oracle.cpu_threads()
    done, t0 = 0, time.perf_counter()
    while done < max_spp:
        oracle.render_stock(ref, cam, st, first + done, 1, threads)
        done += 1
        if time.perf_counter() - t0 >= min_seconds:
            break
    dt = time.perf_counter() - t0
    return st.width * st.height * done / dt, threads, done, dt


def run_reference(args):
    """The reference's own CPU implementation of the path (Renderer::renderSamples of the
    reference sources, built with its shipping flags) on the same workload and step: no product
    module or library is loaded in this process."""
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    if not oracle.available(fast=True):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libphoton_ref_fast.so was not built"}))
        return 0
    desc = workload_description()
    ref = oracle.ref_scene_from_description(desc, fast=True)
    cam = oracle.DescCamera(desc["camera"], fast=True)
    st = oracle.DescSettings(desc["settings"])
    threads = oracle.cpu_threads()
    for w in range(args.warmup):
        oracle.render_stock(ref, cam, st, step_samples(0, 0, w), SPP_PER_STEP, threads)
    t0 = time.perf_counter()
    for k in range(args.steps):
        oracle.render_stock(ref, cam, st, step_samples(0, args.warmup, k), SPP_PER_STEP, threads)
    dt = time.perf_counter() - t0
    value = st.width * st.height * SPP_PER_STEP * args.steps / dt
    sample = f"{args.steps} steps of {SPP_PER_STEP} spp over the full 1920x1080 frame (Renderer::renderSamples)"
    print(json.dumps({
        "impl": "reference", "metric": "paths/s", "value": value, "unit": "paths/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural scene)", "config": workload_config(desc),
        "cpu_baseline": {"value": value, "unit": "paths/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "loaded_libraries": loaded_libraries(),
    }))
    return 0


def loaded_libraries() -> list:
    """Shared objects of this repository mapped into the process."""
    try:
        maps = pathlib.Path("/proc/self/maps").read_text().splitlines()
    except OSError:
        return []
    root = str(ROOT)
    return sorted({line.split()[-1][len(root) + 1:] for line in maps
                   if line.split()[-1].startswith(root) and line.split()[-1].endswith(".so")})


def pe_load():
    import pe_pkg
    return pe_pkg.load()


def run_ours(args):
    world, rank, local = dist_setup()
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    pe = pe_load()
    scene, cam, st, desc = build_workload(pe)
    dev = pe.CudaDevice(local)
    dev.set_scene(scene)
    if args.tuning:
        # fixed knobs instead of the autotuner (for profiler runs, whose timings the tuner cannot trust)
        knobs = [int(v) for v in args.tuning.split(",")]
        closest, anyhit, budget, tail = knobs[:4]
        slots = knobs[4] if len(knobs) > 4 else 1 << 23
        dev.set_tuning(tail_paths=tail, closest_traversal=closest, shade_budget=budget, any_traversal=anyhit,
                       wave_slots=slots)
        tune_log = "fixed by --tuning"
    else:
        dev.autotune(cam, st, SPP_PER_STEP)  # untimed set-up: picks traversal, register budget, tail
        tune_log = dev.autotune_log()
    tuning = dev.tuning()
    tail = tuning["tail_paths"]
    # disjoint sample indices per replica; step k renders samples base + SPP_PER_STEP·(1 + warmup + k) …
    base = replica_sample_base(rank, args.warmup, args.steps)

    # algorithmic bytes per closest-hit ray, counted on the device over one untimed 1-spp pass
    dev.set_counting(True)
    dev.render_resident(cam, st, base, 1)
    cs = dev.last_stats()
    dev.set_counting(False)
    dev.film_clear()
    for w in range(args.warmup):
        dev.render_resident(cam, st, step_samples(base, 0, w), SPP_PER_STEP)
    dev.synchronize()
    if pg:
        import torch
        pg.barrier()
    launches = 0
    rays = 0
    rays_isect = 0
    shadow_rays = 0
    ms_isect = 0.0
    n_isect = 0
    kernel_ms = {"closest_hit": 0.0, "shade": 0.0, "any_hit": 0.0, "tail": 0.0, "total": 0.0}
    with ClockSampler(dev.pci_bus_id) as clocks:
        dev.timer_begin()
        for k in range(args.steps):
            dev.render_resident(cam, st, step_samples(base, args.warmup, k), SPP_PER_STEP)
            s = dev.last_stats()
            launches += s.kernel_launches
            rays += s.closest_rays
            rays_isect += s.closest_rays - s.tail_closest_rays
            shadow_rays += s.shadow_rays
            ms_isect += s.ms_intersect
            n_isect += s.intersect_launches
            for key, v in (("closest_hit", s.ms_intersect), ("shade", s.ms_shade), ("any_hit", s.ms_shadow),
                           ("tail", s.ms_tail), ("total", s.ms_total)):
                kernel_ms[key] += v / args.steps
        ms = dev.timer_end()
    if pg:
        ms = max_over_ranks(ms, pg, f"cuda:{local}")
        pg.barrier()
    total_paths = WIDTH * HEIGHT * SPP_PER_STEP * args.steps * world
    value = total_paths / (ms / 1000.0)

    # end-to-end through RenderDevice::render with host films
    film = pe.Film(WIDTH, HEIGHT)
    for w in range(min(2, args.warmup)):
        dev.render(cam, st, pe.RenderTargets(beauty=film), step_samples(base, 0, w), SPP_PER_STEP)
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        dev.render(cam, st, pe.RenderTargets(beauty=film), step_samples(base, args.warmup, k), SPP_PER_STEP)
    e2e_s = time.perf_counter() - t0
    if pg:
        e2e_s = max_over_ranks(e2e_s, pg, f"cuda:{local}")
    e2e = total_paths / e2e_s

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        dev.close()
        return 0

    # roofline of the closest-hit kernel: per-ray algorithmic bytes from the counting pass
    node_bytes = 64 if tuning["closest_traversal"] == 0 else NODE_BYTES  # binary node 64 B, 4-wide 128 B
    bytes_per_ray = (cs.node_visits * node_bytes + cs.tri_tests * TRI_BYTES) / max(1, cs.closest_rays) + \
        RAY_BYTES + HIT_BYTES + QUEUE_BYTES
    peak, peak_kind = measured_peaks()
    # only the rays the bounce-by-bounce closest-hit launches traced (the tail kernel's are its own)
    achieved = (rays_isect * bytes_per_ray) / (ms_isect / 1000.0) / 1e9 if ms_isect > 0 else None
    traffic = None
    tfile = ROOT / "profiles" / "closest_hit_dram_bytes_per_ray.txt"
    if tfile.exists():
        try:
            per_ray = float(tfile.read_text().split()[0])
            traffic = per_ray * rays_isect / max(1, n_isect)
        except (ValueError, IndexError):
            traffic = None
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "traffic": traffic,
            "kernel": "kIntersect (closest-hit BVH traversal)", "peak_kind": peak_kind,
            "bytes_per_ray": bytes_per_ray, "avg_launch_ms": ms_isect / max(1, n_isect),
            "rays_per_launch": rays_isect / max(1, n_isect)}

    # the shading kernels (one lean kernel per shading key): algorithmic bytes per shaded path —
    # nine 16-byte state columns and the binned slot index in; eight columns out; the hit record's
    # triangle (16 B vertex ids, 3 × 40 B vertex position / normal / uv); one 64-byte shadow record
    # and its 4-byte queue entry per NEE sample; a 4-byte next-queue entry
    shade_bytes = 9 * 16 + 4 + 8 * 16 + 16 + 3 * 40 + 68 * shadow_rays / max(1, rays_isect) + 4
    shade_ms = kernel_ms["shade"] * args.steps
    shade_achieved = (rays_isect * shade_bytes) / (shade_ms / 1000.0) / 1e9 if shade_ms > 0 else None
    roof_shade = {"bound": "hbm", "achieved": shade_achieved, "peak": peak, "unit": "GB/s",
                  "frac": (shade_achieved / peak) if shade_achieved else None, "kernel": "kShadeKey (lean shading)",
                  "peak_kind": peak_kind, "bytes_per_path": shade_bytes,
                  "paths_per_step": rays_isect / args.steps}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            v, threads, done, dt = cpu_reference(desc, args.cpu_seconds, 64, first=100000)
            cpu = {"value": v, "unit": "paths/s", "cores": threads, "kind": "reference",
                   "sample": f"{done} full 1920x1080 frames at 1 spp ({dt:.1f} s), reference shipping build"}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "paths/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}

    out = {
        "metric": "paths/s", "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "config": {**workload_config(desc), "parallelism": f"replicas x{world}"},
        "rays_per_s": (rays + shadow_rays) * world / (ms / 1000.0),
        "closest_rays_per_step": rays / args.steps, "shadow_rays_per_step": shadow_rays / args.steps,
        "e2e": {"value": e2e, "unit": "paths/s", "h2d_bytes_per_step": 76 + 40,
                "d2h_bytes_per_step": WIDTH * HEIGHT * (12 + 4 + 4)},
        "gpu_launches": int(launches),
        "autotuned_tail_paths": tail,
        "tuning": tuning,
        "autotune_log": tune_log.strip().splitlines(),
        "kernel_ms_per_step": kernel_ms,
        "roofline": roof,
        "roofline_shade": roof_shade,
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
    }
    print(json.dumps(out))
    if pg:
        pg.destroy_process_group()
    dev.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tuning", default="",
                    help="closest,any,budget,tail[,wave_slots]: fixed device tuning instead of the autotuner "
                         "(profiler runs)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--serve", action="store_true",
                    help="served-mix benchmark (request server vs the plain per-request loop) instead")
    ap.add_argument("--serve-requests", type=int, default=24)
    ap.add_argument("--serve-quick", action="store_true", help="small scenes (a smoke run of the served mix)")
    ap.add_argument("--guide", action="store_true",
                    help="time to a relMSE target on the indirect-lit room: plain vs learned proposal vs SD-tree")
    ap.add_argument("--profile-case", action="store_true",
                    help="a small case for kernel captures: 960x540 knot waves, then guided room waves")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)
    if args.serve:
        return run_serve(args)
    if args.profile_case:
        return run_profile_case()
    if args.guide:
        return run_guide(args)
    return run_ours(args)


def run_profile_case():
    """Small, fixed launches for ncu captures of single kernels (a few GB on the device): three
    1-spp passes of the knot at 960×540 (≈518 k paths per wave), then four 2-spp passes of the
    room at 320×180 with the learned proposal on (tensor-core inference and training kernels)."""
    pe = pe_load()
    from photon_engine_b200 import scenes
    dev = pe.CudaDevice(0)
    scene, cam, st = scenes.torus_knot_scene(960, 540, 1, 12)
    scene.build_accelerator()
    dev.set_scene(scene)
    times = []
    for k in range(3):
        dev.render_resident(cam, st, k, 1)
        times.append(dev.last_stats().ms_total)
    room, rcam, rst = scenes.room_scene(320, 180, 2, 8, knot_res=(256, 32), env_size=(256, 128))
    room.build_accelerator()
    dev.set_scene(room)
    lib = pe._capi.load()
    pe._capi.check(lib.pe_device_set_guiding(dev.handle, 1, 1, 3e-3))
    film = pe.Film(320, 180)
    for k in range(4):
        dev.render(rcam, rst, pe.RenderTargets(beauty=film), 2 * k, 2)
        times.append(dev.last_stats().ms_total)
    pe._capi.check(lib.pe_device_set_guiding(dev.handle, 0, 0, 0.0))
    print(json.dumps({"profile_case_ms": times}))
    dev.close()
    return 0


def run_serve(args):
    """The served mix on one GPU: request server vs the plain per-request loop (servebench.py)."""
    pe = pe_load()
    from photon_engine_b200 import servebench
    dev = pe.CudaDevice(0)
    with ClockSampler(dev.pci_bus_id) as clocks:
        res = servebench.run(pe, dev, n_requests=args.serve_requests, quick=args.serve_quick)
    s, p = res["served"], res["plain"]
    out = {"metric": "served paths/s (Poisson mix over 4 resident scenes)", "value": s["paths_per_s"],
           "unit": "paths/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
           "data": "synthetic (seeded procedural scenes and request stream)",
           "config": {"workload": "served mix: Cornell / 1M-tri knot / media / 5.2M-tri grid"
                      + (" (reduced scenes)" if args.serve_quick else ""), **res["mix"]},
           "served": s, "plain": p, "served_over_plain": res["speedup"],
           "preview_p99_ms": s["preview_p99_ms"], "clocks": clocks.summary()}
    print(json.dumps(out))
    dev.close()
    return 0


def run_guide(args):
    """Guided sampling's time to a relMSE target against plain sampling (guidebench.py)."""
    pe = pe_load()
    from photon_engine_b200 import guidebench
    dev = pe.CudaDevice(0)
    with ClockSampler(dev.pci_bus_id) as clocks:
        res = guidebench.run(pe, dev)
    out = {"metric": "time-to-relMSE speed-up of guided sampling (indirect-lit room)",
           "value": res["time_to_relmse_speedup"], "unit": "x", "n_gpus": 1, "higher_is_better": True,
           "dtype": "f32", "data": "synthetic (seeded procedural scene)", **res, "clocks": clocks.summary()}
    print(json.dumps(out))
    dev.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
