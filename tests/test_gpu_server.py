"""The request server: continuous batching of many requests into shared waves, admission by an
HBM budget, and results that do not depend on the mix — every request's film equals, bit for
bit, a lone CudaDevice.render of the same samples."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _settings(pe, w, h, depth, filt=None, seed=12345, clamp=0.0):
    st = pe.RenderSettings(width=w, height=h, max_bounces=depth, seed=seed, clamp_indirect=clamp)
    if filt is not None:
        st.filter_type, st.filter_width = filt
    return st


@pytest.fixture(scope="module")
def three_scenes(pe):
    S = scenes()
    c, c_cam, _ = S.cornell_box(64, 64, 8, 8, seed=0)
    k, k_cam, _ = S.torus_knot_scene(96, 54, 4, 12, nu=256, nv=32, env_size=(128, 64))
    m, m_cam, _ = S.media_scene(96, 54, 4, 24, n_leds=200, sphere_res=(32, 16), cyl_res=(24, 4), slab_res=3)
    for sc in (c, k, m):
        sc.build_accelerator()
    return [(c, c_cam), (k, k_cam), (m, m_cam)]


def _lone(pe, device, scene, cam, st, spp):
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, spp)
    return film


def _same(a, b):
    return (np.array_equal(a.sum.view(np.uint32), b.sum.view(np.uint32)) and np.array_equal(a.count, b.count)
            and np.array_equal(a.sum_sq.view(np.uint32), b.sum_sq.view(np.uint32)))


def test_served_films_equal_lone_renders(pe, device, three_scenes):
    PF = pe.PixelFilterType
    reqs = [  # (scene, w, h, depth, filter, seed, clamp, spp, priority)
        (0, 64, 64, 8, None, 0, 0.0, 16, 0),
        (1, 96, 54, 12, None, 12345, 0.0, 6, 0),
        (2, 96, 54, 24, None, 7, 0.0, 4, 0),
        (0, 200, 120, 6, (PF.Box, 1.0), 3, 0.0, 3, 1),
        (1, 2048, 1080, 4, (PF.Gaussian, 2.0), 11, 0.0, 2, 0),   # larger than one wave: split rows
        (1, 160, 90, 12, (PF.Triangle, 1.5), 5, 4.0, 9, 0),
        (2, 64, 36, 24, (PF.Box, 1.0), 1, 0.0, 33, 2),
        (0, 32, 32, 8, None, 99, 0.0, 1, 0),
    ]
    ids = []
    with pe.RenderServer(device, 8 << 30) as srv:
        sid = [srv.add_scene(sc) for sc, _ in three_scenes]
        for (s, w, h, depth, filt, seed, clamp, spp, prio) in reqs:
            st = _settings(pe, w, h, depth, filt, seed, clamp)
            ids.append(srv.submit(sid[s], three_scenes[s][1], st, spp, prio))
        films = []
        for rid in ids:
            assert srv.wait(rid, 300000)
            films.append(srv.take(rid))
        stats = srv.stats()
    assert stats.completed == len(reqs) and stats.failed == 0
    assert stats.segments > stats.waves  # requests shared waves
    for (s, w, h, depth, filt, seed, clamp, spp, prio), film in zip(reqs, films):
        st = _settings(pe, w, h, depth, filt, seed, clamp)
        lone = _lone(pe, device, three_scenes[s][0], three_scenes[s][1], st, spp)
        assert _same(film, lone), (s, w, h, spp)


def test_admission_waits_for_budget(pe, device, three_scenes):
    scene, cam = three_scenes[0]
    st = _settings(pe, 256, 256, 8)
    film_bytes = 256 * 256 * 20
    with pe.RenderServer(device, 1 << 30) as srv:
        sid = srv.add_scene(scene)
        scene_bytes = srv.stats().scene_bytes
        srv.close()
    # room for two films at a time
    with pe.RenderServer(device, scene_bytes + 2 * film_bytes + 1024) as srv:
        sid = srv.add_scene(scene)
        ids = [srv.submit(sid, cam, st, 4) for _ in range(6)]
        for rid in ids:
            assert srv.wait(rid, 120000)
            srv.take(rid)
        s = srv.stats()
    assert s.completed == 6
    assert s.film_bytes_peak <= 2 * film_bytes


def test_smaller_request_finishes_first(pe, device, three_scenes):
    scene, cam = three_scenes[1]
    with pe.RenderServer(device, 4 << 30) as srv:
        sid = srv.add_scene(scene)
        big = srv.submit(sid, cam, _settings(pe, 512, 512, 12), 256)
        small = srv.submit(sid, cam, _settings(pe, 64, 64, 12), 4)
        assert srv.wait(small, 120000) and srv.wait(big, 300000)
        a, b = srv.status(small), srv.status(big)
        srv.take(small)
        srv.take(big)
    assert a.done_ms < b.done_ms


def test_film_larger_than_budget_is_rejected(pe, device, three_scenes):
    scene, cam = three_scenes[0]
    with pe.RenderServer(device, 64 << 20) as srv:
        sid = srv.add_scene(scene)
        with pytest.raises(pe._capi.PhotonError):
            srv.submit(sid, cam, _settings(pe, 4096, 4096, 8), 1)
