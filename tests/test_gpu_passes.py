"""Render passes (RenderPassFilms, renderer.h:59-98) on the CUDA path against the reference
engine's Renderer::renderSamples with passes (renderer.cpp:392-531; crediting in
PathTracer::Li, path_tracer.cpp:373-395, 487-511, 555-590, 676-695, 797-812) on the scene of the
reference's own pass test (test_render_passes.cpp:33-55: a floor, a metal and a glass sphere, a
visible emitter, an area light, a uniform sky), same Owen-Sobol indices (seed 12345):

* the eight light passes match the reference's and sum to the beauty film in every pixel
  (test_render_passes.cpp:77-86, worst relative gap < 1e-4);
* each lobe group lands where that test expects it (metal → glossy, the sky → background, the
  emitter → emission, glass → transmission);
* depth, position and object id (idColor of the node uid) match the reference's; the material id
  colour is the reference's function of a per-material id (the reference hashes the material's
  address, so its colours differ from run to run);
* light groups: "Default" for the emitter's triangles, the area light's and the sky's own, each
  matching the reference's and summing to the beauty film.

Tolerance: the beauty film is bit-exact against the reference at equal spp, so every pass is
held to relMSE ≤ 1e-6 against the reference's (measured on B200: see the asserts).
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _pass_scene(pe, groups=False):
    S = scenes()
    scene = pe.Scene()
    up = (0.0, 1.0, 0.0)
    floor = np.array([[-4, 0, -4], [4, 0, -4], [4, 0, 4], [-4, 0, 4]], np.float32)
    scene.add_shape(pe.TriangleMesh(floor, np.array([up] * 4, np.float32), None, np.array([0, 2, 1, 0, 3, 2]),
                                    pe.Lambertian((0.6, 0.6, 0.6))))
    p, n, i = S.uv_sphere((-0.8, 0.6, 0.0), 0.6, 48, 24)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, pe.DisneyMaterial((0.95, 0.8, 0.5), 1.0, 0.25, 0.5)))
    metal = scene.shape_count() - 1
    p, n, i = S.uv_sphere((0.8, 0.6, 0.0), 0.6, 48, 24)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, pe.Dielectric(1.5, (1.0, 1.0, 1.0))))
    glass = scene.shape_count() - 1
    ep = np.array([[-0.4, 1.8, -1.5], [0.4, 1.8, -1.5], [0.4, 2.4, -1.5], [-0.4, 2.4, -1.5]], np.float32)
    scene.add_shape(pe.TriangleMesh(ep, None, None, np.array([0, 1, 2, 0, 2, 3]),
                                    pe.Lambertian((0.0, 0.0, 0.0), emission=(6.0, 6.0, 6.0))))
    key = pe.AreaLight((-2.0, 3.0, 1.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), (8.0, 8.0, 8.0))
    scene.add_light(key)
    sky = pe.EnvironmentLight(None, 0.0, 0.4)
    scene.set_environment(sky)
    if groups:
        key.set_light_group("Key")
        sky.set_light_group("Sky")
    for k, uid in ((0, 11), (metal, 22), (glass, 33)):
        scene.tag_shape(k, uid)
    cam = pe.PerspectiveCamera((0.0, 1.4, 4.5), (0.0, 0.8, 0.0), up, 45.0, 4.0 / 3.0)
    st = pe.RenderSettings(width=64, height=48, max_bounces=6, seed=12345)
    return scene, cam, st


def _render(pe, device, scene, cam, st, spp):
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    passes = pe.RenderPassFilms(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film, passes=passes), 0, spp)
    return film, passes


def _worst_gap(parts, beauty):
    s = np.sum(parts, axis=0)
    return float(np.max(np.abs(s - beauty) / np.maximum(1.0, beauty)))


def test_light_passes_match_reference_and_sum_to_beauty(pe, device, oracle):
    scene, cam, st = _pass_scene(pe)
    spp = 16
    film, passes = _render(pe, device, scene, cam, st, spp)
    mean, cnt, light, data, groups = oracle.RefScene(scene).render_passes(cam, st, 0, spp)
    assert np.array_equal(film.count, cnt)
    beauty = film.resolve()
    assert pe.rel_mse(beauty, mean) < 1e-6
    mine = [f.resolve() for f in passes.light]
    for k in range(8):
        assert np.array_equal(passes.light[k].count, cnt)
        err = pe.rel_mse(mine[k], light[k])
        assert err < 1e-6, (pe.LightPass(k).name, err)
    # the passes rebuild the beauty film (test_render_passes.cpp:77-86)
    assert _worst_gap(mine, beauty) < 1e-4
    tot = {p: float(mine[p].sum()) for p in pe.LightPass}
    for p in (pe.LightPass.DiffuseDirect, pe.LightPass.DiffuseIndirect, pe.LightPass.GlossyDirect,
              pe.LightPass.TransmissionIndirect, pe.LightPass.Emission, pe.LightPass.Background):
        assert tot[p] > 0.0, p.name
    # the metal sphere's centre is glossy, not diffuse (test_render_passes.cpp:97-104)
    my, mx = int(0.52 * st.height), int(0.37 * st.width)
    lum = lambda im: float(im[my, mx] @ np.array([0.2126, 0.7152, 0.0722], np.float32))
    gloss = lum(mine[pe.LightPass.GlossyDirect]) + lum(mine[pe.LightPass.GlossyIndirect])
    diff = lum(mine[pe.LightPass.DiffuseDirect]) + lum(mine[pe.LightPass.DiffuseIndirect])
    assert gloss > 10.0 * diff + 1e-4, (gloss, diff)
    # data passes: depth near the camera distance, position and object ids as the reference's
    depth = passes.depth.resolve()
    assert abs(float(depth[my, mx, 0]) - 4.0) < 0.6
    for name, m, r in (("depth", depth, data[0]), ("position", passes.position.resolve(), data[1]),
                       ("object_id", passes.object_id.resolve(), data[2])):
        same = float(np.mean(np.all(np.abs(m - r) <= 1e-5 * np.maximum(1.0, np.abs(r)), axis=-1)))
        assert same > 0.995, (name, same)
    # every hit pixel carries a material colour; the sky carries none
    mat = passes.material_id.resolve()
    assert np.all(mat[depth[..., 0] > 0].max(axis=-1) > 0.0)
    assert np.all(mat[depth[..., 0] == 0] == 0.0)


def test_light_groups_match_reference(pe, device, oracle):
    scene, cam, st = _pass_scene(pe, groups=True)
    spp = 8
    film, passes = _render(pe, device, scene, cam, st, spp)
    names = [n for n, _ in passes.light_groups]
    assert sorted(names) == ["Default", "Key", "Sky"], names
    assert names == scene.light_group_names()
    mean, cnt, light, data, groups = oracle.RefScene(scene).render_passes(cam, st, 0, spp)
    assert len(groups) == 3
    beauty = film.resolve()
    mine = [f.resolve() for _, f in passes.light_groups]
    for g in range(3):
        assert pe.rel_mse(mine[g], groups[g]) < 1e-6, names[g]
        assert float(mine[g].sum()) > 0.0, names[g]
    # the groups rebuild the beauty film too
    assert _worst_gap(mine, beauty) < 1e-4


def test_passes_with_aovs_and_across_batches(pe, device):
    """Passes and AOVs of one call; two batches of 4 spp equal one of 8 (films accumulate)."""
    scene, cam, st = _pass_scene(pe)
    scene.build_accelerator()
    device.set_scene(scene)
    one = pe.RenderPassFilms(st.width, st.height)
    aovs = pe.AovFilms(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=pe.Film(st.width, st.height), aovs=aovs, passes=one), 0, 8)
    assert int(aovs.alpha.count.min()) == 8
    two = pe.RenderPassFilms(st.width, st.height)
    film = pe.Film(st.width, st.height)
    for s0 in (0, 4):
        device.render(cam, st, pe.RenderTargets(beauty=film, passes=two), s0, 4)
    for a, b in zip(one.light, two.light):
        assert np.array_equal(a.count, b.count)
        np.testing.assert_allclose(a.resolve(), b.resolve(), rtol=1e-5, atol=1e-6)
    # a session with SessionConfig.passes keeps them (render_session.h:75)
    sess = pe.RenderSession(device)
    sess.begin(cam, st, pe.SessionConfig(passes=True, target_spp=4))
    while sess.advance():
        pass
    assert sess.passes is not None and not sess.warnings
    assert int(sess.passes.light[0].count.min()) == 4


def test_cryptomatte_matches_reference(pe, device, oracle):
    """CryptoObject / CryptoMaterial (CryptoFilm, cryptomatte.cpp; ids of the first hit,
    renderer.cpp:170-175, named as buildCryptoLookup names them, renderer.cpp:75-118): per pixel
    the same ids with the same coverage as the reference's pixelRanks."""
    scene, cam, st = _pass_scene(pe)
    scene.set_shape_name(0, "Floor")
    metal = scene.ops[1][1].material
    scene.set_material_name(metal, "BrushedGold")
    scene.build_accelerator()
    device.set_scene(scene)
    spp = 8
    passes = pe.RenderPassFilms(st.width, st.height)
    passes.enable_cryptomatte()
    device.render(cam, st, pe.RenderTargets(beauty=pe.Film(st.width, st.height), passes=passes), 0, spp)
    ref = oracle.RefScene(scene).render_crypto(cam, st, 0, spp)
    worst = 0.0
    ids = set()
    for f, film in enumerate((passes.crypto_object, passes.crypto_material)):
        for y in range(st.height):
            for x in range(st.width):
                mine = dict(film.pixel_ranks(x, y))
                theirs = {float(i): float(c) for i, c in ref[f, y, x] if c > 0.0}
                assert set(mine) == set(theirs), (f, x, y, mine, theirs)
                for i, c in theirs.items():
                    worst = max(worst, abs(mine[i] - c))
                ids.update(mine)
    assert worst < 1e-6, worst
    # floor, metal, glass, emitter and the sky-free pixels give several distinct ids
    assert len(ids) >= 6, ids
