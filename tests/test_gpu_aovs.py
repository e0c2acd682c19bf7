"""The AOV films (AovFilms, renderer.h:42-53) on the CUDA path against the reference engine's
Renderer::renderSamples with AOVs (renderer.cpp:392-531, tracePixel 139-204, addAovs 219-224)
on the same scenes and Owen-Sobol indices (seed 12345):

* albedo: the first visible surface's base colour clamped to [0, 1], or the background seen by a
  camera ray that misses (its colour, or the environment in that direction);
* normal: that surface's normal, summed signed;
* alpha: 1 on a hit, 0 on a miss, what thin glass holds back in front of a transparent
  background, and the shadow's opacity on a shadow catcher over a transparent background.

Tolerance: the AOVs come from the camera ray's first hit, so they are equal to the reference's
except where a filter or lens warp (cosf / sinf, an ulp apart between CUDA and glibc) moves a
sample across a silhouette: ≥ 99.5 % of the pixels equal to 1e-5, mean absolute difference
≤ 1e-3 (measured on B200: every pixel equal, mean difference ≤ 3e-9).  The beauty film at equal
spp is held to relMSE ≤ 1e-4 as in the other parity tests (measured: ≤ 2e-13).
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _open_scene(pe, mode):
    S = scenes()
    scene = pe.Scene()
    gp, gi = S._wall_grid((-4.0, 0.0, 4.0), (8.0, 0.0, 0.0), (0.0, 0.0, -8.0), 4, 4, None)
    scene.add_shape(pe.TriangleMesh(gp, None, None, gi, pe.Lambertian((0.5, 0.5, 0.5))))
    ground = scene.shape_count() - 1
    p, n, i = S.uv_sphere((-0.9, 0.7, 0.0), 0.7, 48, 24)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, pe.DisneyMaterial((1.4, 0.3, 0.2), 0.0, 0.4, 0.5)))
    p, n, i = S.uv_sphere((0.9, 0.6, 0.3), 0.6, 48, 24)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, pe.Mirror((0.9, 0.8, 0.7))))
    # a thin-walled glass pane in front of the spheres, part of it over the background
    glass = pe.Dielectric(1.5, (0.9, 0.95, 1.0))
    glass.set_thin_walled(True)
    pp, pi = S._wall_grid((-0.3, 0.2, -1.5), (1.8, 0.0, 0.0), (0.0, 2.4, 0.0), 2, 2, None)
    scene.add_shape(pe.TriangleMesh(pp, None, None, pi, glass))
    scene.add_light(pe.AreaLight((-1.0, 4.0, -1.0), (2.0, 0.0, 0.0), (0.0, 0.0, 2.0), (20.0, 20.0, 20.0)))
    if mode == "environment":
        sky = np.ones((32, 64, 3), np.float32) * np.linspace(0.2, 1.6, 32, dtype=np.float32)[:, None, None]
        scene.set_environment(pe.EnvironmentLight(sky, 0.0, 1.0))
    elif mode == "color":
        scene.set_background(pe.Background(pe.BackgroundMode.Color, (0.3, 0.4, 0.5)))
    else:
        scene.set_background(pe.Background(pe.BackgroundMode.Transparent))
    if mode == "catcher":
        scene.set_shadow_catcher(ground)
    cam = pe.PerspectiveCamera((0.0, 1.6, -5.0), (0.0, 0.6, 0.0), (0.0, 1.0, 0.0), 45.0, 1.0)
    # Renderer::renderSamples seeds its sampler with 12345 (renderer.cpp:437)
    st = pe.RenderSettings(width=64, height=64, max_bounces=6, seed=12345)
    return scene, cam, st


def _agree(a, b):
    same = float(np.mean(np.all(np.abs(a - b) <= 1e-5 * np.maximum(1.0, np.abs(b)), axis=-1)))
    return same, float(np.mean(np.abs(a - b)))


@pytest.mark.parametrize("mode", ["color", "transparent", "environment", "catcher"])
def test_aovs_match_reference(pe, device, oracle, mode):
    scene, cam, st = _open_scene(pe, mode)
    scene.build_accelerator()
    device.set_scene(scene)
    spp = 8
    film = pe.Film(st.width, st.height)
    aovs = pe.AovFilms(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film, aovs=aovs), 0, spp)
    ref = oracle.RefScene(scene)
    beauty, albedo, normal, alpha, cnt, acnt = ref.render_aovs(cam, st, 0, spp)
    assert np.array_equal(film.count, cnt)
    for f in (aovs.albedo, aovs.normal, aovs.alpha):
        assert np.array_equal(f.count, acnt)
    err = pe.rel_mse(film.resolve(), beauty)
    assert err < 1e-4, err
    for name, mine, theirs in (("albedo", aovs.albedo, albedo), ("normal", aovs.normal, normal),
                               ("alpha", aovs.alpha, alpha)):
        same, mad = _agree(mine.resolve(), theirs)
        assert same > 0.995 and mad < 1e-3, (name, same, mad)
    a = aovs.alpha.resolve()[..., 0]
    if mode in ("transparent", "catcher"):
        # partial coverage somewhere: behind the glass pane, or the catcher's shadow
        assert np.any((a > 0.02) & (a < 0.98)), mode
    if mode in ("color", "transparent", "environment"):
        # the background shows beside the objects: some pixels miss with every sample
        assert np.mean(a == 0.0) > 0.05, np.mean(a == 0.0)
    # the albedo of the red sphere is clamped to 1
    assert aovs.albedo.resolve().max() <= 1.0 + 1e-6


def test_aovs_across_batches_equal_one_batch(pe, device):
    """Films accumulate: two batches of 4 spp give the AOV films of one batch of 8."""
    scene, cam, st = _open_scene(pe, "transparent")
    scene.build_accelerator()
    device.set_scene(scene)
    one = pe.AovFilms(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=pe.Film(st.width, st.height), aovs=one), 0, 8)
    two = pe.AovFilms(st.width, st.height)
    beauty = pe.Film(st.width, st.height)
    for s0 in (0, 4):
        device.render(cam, st, pe.RenderTargets(beauty=beauty, aovs=two), s0, 4)
    for a, b in ((one.albedo, two.albedo), (one.normal, two.normal), (one.alpha, two.alpha)):
        assert np.array_equal(a.count, b.count)
        np.testing.assert_allclose(a.resolve(), b.resolve(), rtol=1e-5, atol=1e-6)


def test_session_keeps_aovs(pe, device):
    """RenderSession with SessionConfig.aovs hands the AOV films to every batch (render_session.h:74)."""
    scene, cam, st = _open_scene(pe, "color")
    scene.build_accelerator()
    device.set_scene(scene)
    sess = pe.RenderSession(device)
    sess.begin(cam, st, pe.SessionConfig(aovs=True, target_spp=6))
    while sess.advance():
        pass
    assert sess.samples == 6
    aovs = sess.aovs
    assert aovs is not None and not sess.warnings
    assert int(aovs.alpha.count.min()) == 6
    a = aovs.alpha.resolve()[..., 0]
    assert a.max() == 1.0 and a.min() == 0.0
