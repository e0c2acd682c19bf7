"""Light linking and shadow linking (Light::setLightLink, Scene::tagShape; path_tracer.cpp:536-537,
571-572, 641-644 and the shadow walk of :172-202) on the CUDA path against the reference engine's
CPU path on the same scene and Owen-Sobol indices: a light that only lights some tagged objects, a
light that skips the floor, and a blocker whose shadow one light ignores.

Tolerance as for the other equal-spp scene tests: relMSE ≤ 1e-4, ≥ 99 % of the pixels equal to
1e-4 relative, no bias."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene(pe, links: bool):
    S = importlib.import_module("photon_engine_b200.scenes")
    scene = pe.Scene()
    white = pe.Lambertian((0.7, 0.7, 0.7))
    fp, fi = S._wall_grid((-4.0, 0.0, 4.0), (8.0, 0.0, 0.0), (0.0, 0.0, -8.0), 4, 4, None)
    scene.add_shape(pe.TriangleMesh(fp, None, None, fi, white))                    # shape 0: floor
    bp, bi = S._wall_grid((-4.0, 0.0, 3.0), (0.0, 4.0, 0.0), (8.0, 0.0, 0.0), 4, 4, None)
    scene.add_shape(pe.TriangleMesh(bp, None, None, bi, white))                    # shape 1: back wall
    p, n, i = S.grid_box((-1.2, 0.6, 0.5), (1.2, 1.2, 1.2), 2)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, pe.Lambertian((0.8, 0.4, 0.3))))  # shape 2: box A
    p, n, i = S.grid_box((1.2, 0.9, 0.0), (0.8, 1.8, 0.8), 2)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, pe.Lambertian((0.3, 0.6, 0.8))))  # shape 3: box B
    p, n, i = S.uv_sphere((0.2, 0.5, -1.0), 0.5, 32, 16)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, pe.DisneyMaterial((0.9, 0.9, 0.3), 0.0, 0.3, 0.5)))  # 4
    scene.add_light(pe.AreaLight((-3.0, 3.5, -2.0), (1.5, 0.0, 0.0), (0.0, 0.0, 1.5), (18.0, 14.0, 10.0)))  # light 0
    scene.add_light(pe.AreaLight((1.5, 3.5, -2.0), (1.5, 0.0, 0.0), (0.0, 0.0, 1.5), (8.0, 12.0, 18.0)))    # light 1
    scene.set_background(pe.Background(pe.BackgroundMode.Color, (0.05, 0.05, 0.06)))
    if links:
        for shape, uid in ((0, 10), (2, 20), (3, 30), (4, 40)):
            scene.tag_shape(shape, uid)
        scene.set_light_link(0, mode=1, uids=(20, 40), shadow_mode=2, shadow_uids=(30,))
        scene.set_light_link(1, mode=2, uids=(10,))
    cam = pe.PerspectiveCamera((0.0, 2.5, -6.0), (0.0, 0.8, 0.0), (0.0, 1.0, 0.0), 45.0, 1.0)
    st = pe.RenderSettings(width=64, height=64, max_bounces=6, seed=3)
    scene.build_accelerator()
    return scene, cam, st


def _render(pe, device, scene, cam, st, spp):
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, spp)
    return film


def test_light_links_match_reference(pe, device, oracle):
    scene, cam, st = _scene(pe, links=True)
    film = _render(pe, device, scene, cam, st, 8)
    ref, cnt = oracle.RefScene(scene).render(cam, st, 0, 8)
    assert np.array_equal(film.count, cnt)
    img = film.resolve()
    err = pe.rel_mse(img, ref)
    same = np.mean(np.all(np.abs(img - ref) <= 1e-4 * np.maximum(1.0, np.abs(ref)), axis=-1))
    bias = float(img.mean() / ref.mean() - 1.0)
    assert err < 1e-4 and same > 0.99 and abs(bias) < 1e-3, (err, same, bias)
    # the links change the picture: the floor loses light 1 and light 0's light
    plain_scene, _, _ = _scene(pe, links=False)
    plain = _render(pe, device, plain_scene, cam, st, 8).resolve()
    floor = (slice(52, 64), slice(0, 64))
    assert img[floor].mean() < 0.8 * plain[floor].mean(), (img[floor].mean(), plain[floor].mean())
