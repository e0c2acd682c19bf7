"""The parts of PathTracer::Li that cast rays of their own at a surface hit, on the CUDA path
against the reference engine's CPU path on the same scenes and Owen-Sobol indices:

* contact ambient occlusion at camera hits (RenderSettings::aoStrength, approxAo,
  path_tracer.cpp:27-45, 618-621);
* rounded edges (Material::setRoundEdgeRadius, roundedEdgeNormal, path_tracer.cpp:209-255,
  612-615);
* the shadow catcher (Scene::setShadowCatcher, path_tracer.cpp:515-563), under an area light
  and under the environment with its sun.

Tolerance: the disk and hemisphere warps call cosf / sinf, where CUDA and glibc differ by an ulp
or two, so a probe ray can graze an edge differently; images at equal spp agree to relMSE
≤ 1e-4 with ≥ 99 % of the pixels equal to 1e-4 relative, and without bias.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _compare(pe, device, oracle, scene, cam, st, spp):
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, spp)
    ref = oracle.RefScene(scene)
    mean_ref, cnt_ref = ref.render(cam, st, 0, spp)
    assert np.array_equal(film.count, cnt_ref)
    img = film.resolve()
    err = pe.rel_mse(img, mean_ref)
    same = np.mean(np.all(np.abs(img - mean_ref) <= 1e-4 * np.maximum(1.0, np.abs(mean_ref)), axis=-1))
    bias = float(img.mean() / max(1e-12, mean_ref.mean()) - 1.0)
    return img, mean_ref, err, same, bias


def _check(err, same, bias):
    assert err < 1e-4, (err, same, bias)
    assert same > 0.99, (err, same, bias)
    assert abs(bias) < 1e-3, (err, same, bias)


def test_contact_ao_matches_reference(pe, device, oracle):
    S = scenes()
    scene, cam, st = S.cornell_box(64, 64, 8, 8, seed=0)
    st.ao_strength = 0.8
    img, ref, err, same, bias = _compare(pe, device, oracle, scene, cam, st, 8)
    _check(err, same, bias)
    # the AO darkens the image against the same frame without it
    st.ao_strength = 0.0
    device.set_scene(scene)
    plain = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=plain), 0, 8)
    assert img.mean() < 0.995 * plain.resolve().mean()


def test_rounded_edges_match_reference(pe, device, oracle):
    S = scenes()
    scene, cam, st = S.cornell_box(64, 64, 8, 8, seed=0)
    m = pe.Lambertian((0.6, 0.6, 0.7))
    m.set_round_edge_radius(0.25)
    p, n, i = S.grid_box((2.2, 0.8, 2.0), (1.6, 1.6, 1.6), 2)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, m))
    img, ref, err, same, bias = _compare(pe, device, oracle, scene, cam, st, 8)
    _check(err, same, bias)


@pytest.mark.parametrize("light", ["area", "environment"])
def test_shadow_catcher_matches_reference(pe, device, oracle, light):
    S = scenes()
    scene = pe.Scene()
    ground = pe.Lambertian((0.5, 0.5, 0.5))
    gp, gi = S._wall_grid((-4.0, 0.0, 4.0), (8.0, 0.0, 0.0), (0.0, 0.0, -8.0), 4, 4, None)
    scene.add_shape(pe.TriangleMesh(gp, None, None, gi, ground))
    catcher = scene.shape_count() - 1
    p, n, i = S.uv_sphere((0.0, 0.8, 0.0), 0.8, 48, 24)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, pe.DisneyMaterial((0.8, 0.3, 0.2), 0.0, 0.4, 0.5)))
    if light == "area":
        scene.add_light(pe.AreaLight((-1.0, 4.0, -1.0), (2.0, 0.0, 0.0), (0.0, 0.0, 2.0), (20.0, 20.0, 20.0)))
        scene.set_background(pe.Background(pe.BackgroundMode.Color, (0.3, 0.4, 0.5)))
    else:
        sky = np.ones((32, 64, 3), np.float32) * np.linspace(0.2, 1.0, 32, dtype=np.float32)[:, None, None]
        env = pe.EnvironmentLight(sky, 0.0, 1.0)
        env.set_sun((0.4 / 0.943, 0.8 / 0.943, 0.3 / 0.943), 0.999, (40.0, 38.0, 35.0))
        scene.set_environment(env)
    scene.set_shadow_catcher(catcher)
    cam = pe.PerspectiveCamera((0.0, 2.0, -5.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 40.0, 1.0)
    st = pe.RenderSettings(width=64, height=64, max_bounces=6, seed=7)
    img, ref, err, same, bias = _compare(pe, device, oracle, scene, cam, st, 8)
    _check(err, same, bias)
    # the sphere's shadow darkens the caught ground: somewhere below the sphere the image is
    # well under the background seen elsewhere on the ground
    lo = float(np.percentile(img[40:, :].mean(axis=-1), 5))
    hi = float(np.percentile(img[40:, :].mean(axis=-1), 95))
    assert lo < 0.7 * hi, (lo, hi)
