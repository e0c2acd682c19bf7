"""Ray queries against the reference's Scene::intersect / intersectAny (bvh.cpp:322-446,
mesh_instance.cpp:104-123) on the same scene: seeded rays through the scene's box and shadow
rays from the ground towards the area light, over triangles, spheres, mesh instances (static and
moving, at several shutter times) and the visibility masks.

Tolerance: closest hits on the binary tree (the reference's visiting order): shape, triangle and
distance bit-exact; on the 4-wide tree: distances bit-exact (a bit-identical tie may name the
other triangle); any-hit answers identical.  A sphere hit's triangle number is not compared: the
reference's Sphere::intersect leaves SurfaceInteraction::primIndex as an earlier candidate of the
same traversal set it (an instance's triangle), which nothing downstream reads for spheres.
"""
import importlib
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PROJECT = pathlib.Path(__file__).resolve().parent / "golden" / "studio.photon"


def helpers():
    return importlib.import_module("test_instances")


def rays_through(lo, hi, n, seed):
    rng = np.random.default_rng(seed)
    span = hi - lo
    o = lo - 0.5 * span + rng.random((n, 3)) * 2.0 * span
    target = lo + rng.random((n, 3)) * span
    d = target - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.where(rng.random(n) < 0.3, rng.random(n) * np.linalg.norm(span), 1e30)
    return o.astype(np.float32), d.astype(np.float32), tmax.astype(np.float32)


def shadow_rays(light_pos, light_u, light_v, lo, hi, n, seed):
    rng = np.random.default_rng(seed)
    p = lo + rng.random((n, 3)) * (hi - lo)
    p[:, 1] = lo[1] + 1e-3
    q = np.asarray(light_pos) + rng.random((n, 1)) * np.asarray(light_u) + rng.random((n, 1)) * np.asarray(light_v)
    d = q - p
    dist = np.linalg.norm(d, axis=1)
    return p.astype(np.float32), (d / dist[:, None]).astype(np.float32), (dist * 0.999).astype(np.float32)


def sphere_shapes(scene):
    out, shape = [], 0
    for kind, _ in scene.ops:
        if kind == "sphere":
            out.append(shape)
        shape += 2 if kind == "area" else 1
    return np.array(out, np.int32)


def check_queries(device, ref, o, d, tm, mask=0x1F, time=0.0, spheres=()):
    rs, rp, rt = ref.trace_rays(o, d, tm, 0, mask, time)
    ms, mp, mt = device.trace_rays(o, d, tm, 0, mask, time)
    assert np.array_equal(ms, rs), (int((ms != rs).sum()), np.nonzero(ms != rs)[0][:8])
    tri = ~np.isin(rs, np.asarray(spheres, np.int32))
    assert np.array_equal(mp[tri], rp[tri]), (int((mp[tri] != rp[tri]).sum()))
    assert np.array_equal(mt.view(np.uint32), rt.view(np.uint32))
    ws, _, wt = device.trace_rays(o, d, tm, 1, mask, time)
    assert np.array_equal(wt.view(np.uint32), rt.view(np.uint32))
    assert np.array_equal(ws >= 0, rs >= 0)
    ra, _, _ = ref.trace_rays(o, d, tm, 2, mask, time)
    ma, _, _ = device.trace_rays(o, d, tm, 2, mask, time)
    assert np.array_equal(ma, ra), (int((ma != ra).sum()), np.nonzero(ma != ra)[0][:8])
    return rs


def scene_box(scene):
    import ctypes as C
    lib = importlib.import_module("photon_engine_b200")._capi.load()
    b = np.empty(6, np.float32)
    lo, hi = np.full(3, np.inf), np.full(3, -np.inf)
    for i in range(scene.shape_count()):
        lib.pe_scene_shape_bounds(scene.handle, i, b.ctypes.data_as(C.POINTER(C.c_float)))
        if np.all(np.isfinite(b)) and np.all(np.abs(b) < 50):
            lo, hi = np.minimum(lo, b[:3]), np.maximum(hi, b[3:])
    return lo, hi


def test_project_rays_match_reference(pe, device, oracle):
    proj = importlib.import_module("photon_engine_b200.project")
    scene, cam, st = proj.load_project(PROJECT, 96, 72, 4)
    scene.build_accelerator()
    device.set_scene(scene)
    ref = oracle.RefScene(scene)
    lo, hi = scene_box(scene)
    o, d, tm = rays_through(lo, hi, 20000, 1)
    sph = sphere_shapes(scene)
    hit = check_queries(device, ref, o, d, tm, spheres=sph)
    assert (hit >= 0).mean() > 0.3
    area = next(obj for kind, obj in scene.ops if kind == "area")
    o, d, tm = shadow_rays(area.position, area.u, area.v, lo, hi, 20000, 2)
    check_queries(device, ref, o, d, tm, mask=16, spheres=sph)


def test_instanced_cornell_rays_match_reference(pe, device, oracle):
    scene, cam, st = helpers().instanced_cornell(pe, 32, 32, 4, 4, emissive=True)
    scene.build_accelerator()
    device.set_scene(scene)
    ref = oracle.RefScene(scene)
    lo, hi = scene_box(scene)
    o, d, tm = rays_through(lo, hi, 20000, 3)
    check_queries(device, ref, o, d, tm)
    check_queries(device, ref, o, d, tm, mask=16)


@pytest.mark.parametrize("time", [0.0, 0.3, 0.75, 1.0])
def test_moving_instance_rays_match_reference(pe, device, oracle, time):
    scene, cam, st = helpers().moving_cornell(pe, 32, 32, 4, 4)
    scene.build_accelerator()
    device.set_scene(scene)
    ref = oracle.RefScene(scene)
    lo, hi = scene_box(scene)
    o, d, tm = rays_through(lo, hi, 20000, 4)
    check_queries(device, ref, o, d, tm, time=time)
