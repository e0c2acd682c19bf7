"""The per-thread tail kernel finishes a wave's last paths with the wavefront's own shading code
and shadow rays traced inline, so the film must not depend on where a wave switches to it:
all-wavefront, all-tail and the default switch point give the same film bit for bit."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _films(pe, device, scene, cam, st, spp):
    scene.build_accelerator()
    device.set_scene(scene)
    out = {}
    try:
        for name, tail in (("wavefront", 0), ("tail", 1 << 40), ("mixed", 4096), ("default", -1)):
            device.set_tail_paths(tail)
            film = pe.Film(st.width, st.height)
            device.render(cam, st, pe.RenderTargets(beauty=film), 0, spp)
            out[name] = (film, device.last_stats())
    finally:
        device.set_tail_paths(-1)
    return out


def _assert_same(out):
    a = out["wavefront"][0]
    for name in ("tail", "mixed", "default"):
        b = out[name][0]
        assert np.array_equal(a.sum.view(np.uint32), b.sum.view(np.uint32)), name
        assert np.array_equal(a.sum_sq.view(np.uint32), b.sum_sq.view(np.uint32)), name
        assert np.array_equal(a.count, b.count), name
    assert out["wavefront"][1].tail_paths == 0
    assert out["tail"][1].tail_paths == out["tail"][1].paths
    # the same rays are traced whichever kernel traces them
    for name in ("tail", "mixed"):
        assert out[name][1].closest_rays == out["wavefront"][1].closest_rays
        assert out[name][1].shadow_rays == out["wavefront"][1].shadow_rays


def test_tail_cornell_bit_exact(pe, device):
    scene, cam, st = scenes().cornell_box(64, 64, 8, 8, seed=5)
    _assert_same(_films(pe, device, scene, cam, st, 8))


def test_tail_media_bit_exact(pe, device):
    scene, cam, st = scenes().media_scene(80, 45, 4, 24, n_leds=200, sphere_res=(48, 24), cyl_res=(32, 6), slab_res=4)
    _assert_same(_films(pe, device, scene, cam, st, 4))


def test_tail_knot_bit_exact(pe, device):
    scene, cam, st = scenes().torus_knot_scene(160, 90, 2, 12, nu=512, nv=32, env_size=(256, 128))
    _assert_same(_films(pe, device, scene, cam, st, 2))


def test_tail_paths_setting(device):
    try:
        assert device.tail_paths > 0
        device.set_tail_paths(0)
        assert device.tail_paths == 0
        device.set_tail_paths(12345)
        assert device.tail_paths == 12345
    finally:
        device.set_tail_paths(-1)


def test_autotune_picks_a_threshold_and_keeps_results(pe, device):
    scene, cam, st = scenes().cornell_box(64, 64, 8, 8, seed=5)
    scene.build_accelerator()
    device.set_scene(scene)
    try:
        device.set_tail_paths(0)
        a = pe.Film(st.width, st.height)
        device.render(cam, st, pe.RenderTargets(beauty=a), 0, 8)
        device.set_tail_paths(-1)
        grid = device.tail_paths
        chosen = device.autotune(cam, st, 2)
        assert chosen in (grid // 4, grid // 2, grid, 2 * grid)
        assert device.tail_paths == chosen
        b = pe.Film(st.width, st.height)
        device.render(cam, st, pe.RenderTargets(beauty=b), 0, 8)
        assert np.array_equal(a.sum.view(np.uint32), b.sum.view(np.uint32))
    finally:
        device.set_tail_paths(-1)
