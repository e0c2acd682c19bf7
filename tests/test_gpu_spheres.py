"""Analytic spheres (Sphere, src/geometry/sphere.cpp:12-90) on the CUDA path against the reference
engine's CPU path: the BVH holds each sphere as one primitive beside the triangles, the leaf test
is Sphere::intersect's quadratic (solveQuadratic, src/core/math/utils.h:64-88) and the hit record
its projected point, error bound, faced normal, spherical uv and tangent.

Tolerances: primary-hit shape ids and distances bit-exact (the binary tree in the reference's
order; the 4-wide tree ties allowed, as for triangles); images at equal spp relMSE ≤ 1e-4 with
≥ 99 % of pixels equal to 1e-4 relative (the spherical uv uses acos/atan2, CUDA's versus glibc's).
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def sphere_scene(pe, w=96, h=96, spp=8, depth=8):
    S = importlib.import_module("photon_engine_b200.scenes")
    scene, cam, st = S.cornell_box(w, h, spp, depth, seed=3)
    tex = np.kron(np.random.default_rng(4).uniform(0.1, 0.9, (4, 8, 3)).astype(np.float32), np.ones((8, 8, 1), np.float32))
    textured = pe.DisneyMaterial((0.8, 0.8, 0.8), 0.0, 0.35)
    textured.set_albedo_image(tex)
    glass = pe.Dielectric(1.5)
    scene.add_shape(pe.Sphere((1.4, 0.7, 1.2), 0.7, textured))               # uv from the sphere's angles
    scene.add_shape(pe.Sphere((3.9, 0.6, 2.2), 0.6, glass))                  # refraction through a sphere
    scene.add_shape(pe.Sphere((2.8, 2.2, 3.6), 0.45, pe.Mirror((0.9, 0.9, 0.9))))
    scene.add_shape(pe.Sphere((2.2, 4.2, 1.0), 0.3, pe.Lambertian((0.2, 0.5, 0.8))))
    return scene, cam, st


def test_sphere_primary_hits_match_reference(pe, device, oracle):
    scene, cam, st = sphere_scene(pe)
    scene.build_accelerator()
    device.set_scene(scene)
    ref = oracle.RefScene(scene)
    for s in (0, 3):
        rs, rp, rt = ref.trace_primary(cam, st, s)
        ms, mp, mt = device.trace_primary(cam, st, s, ordered=True)
        assert np.array_equal(ms, rs) and np.array_equal(mp, rp)
        assert np.array_equal(mt.view(np.uint32), rt.view(np.uint32))
        assert (ms >= scene.shape_count() - 4).any(), "no sphere seen"
        ws, wp, wt = device.trace_primary(cam, st, s)
        assert np.array_equal(wt.view(np.uint32), rt.view(np.uint32))


def test_sphere_image_matches_reference_at_equal_spp(pe, device, oracle):
    scene, cam, st = sphere_scene(pe)
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, 8)
    mean_ref, cnt_ref = oracle.RefScene(scene).render(cam, st, 0, 8)
    assert np.array_equal(film.count, cnt_ref)
    img = film.resolve()
    err = pe.rel_mse(img, mean_ref)
    same = float(np.mean(np.all(np.abs(img - mean_ref) <= 1e-4 * np.maximum(1.0, np.abs(mean_ref)), axis=-1)))
    assert err <= 1e-4, (err, same)
    assert same >= 0.99, same
