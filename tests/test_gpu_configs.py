"""Parity on the workloads at the sizes their configurations state, against the reference
engine's CPU path on the same scene and Owen-Sobol indices (oracle/_ref, run on this host).

* Plain Cornell box: 256², 64 spp, depth 8, RR after 3, Sobol seed 0 — the whole image at equal
  spp.  Lambert paths use the same arithmetic as the reference; only sin/cos of the cosine lobe
  may differ by an ulp, so the image agrees to relMSE ≤ 1e-6 with ≥ 99 % of pixels equal to
  1e-5 relative.
* The ~1M-triangle torus knot at 1920×1080: primary-hit shape/primitive ids and distances of
  the whole frame bit-exact through the binary tree in the reference's visiting order; through
  the 4-wide tree the render kernels use, distances bit-exact and ids equal except at ties (a
  different triangle at the bit-identical distance: a ray through a shared edge), counted.
* The many-light and media workload at 1280×720 with its 2000 emissive LED triangles (light-BVH
  NEE), dispersive glass, absorbing and scattering volumes and the subsurface slab, depth 24:
  two samples per pixel at equal spp, relMSE ≤ 3e-3 with ≥ 99 % of pixels equal to 1e-4
  relative (a path leaves the reference's only where a transcendental's last ulp flips a
  free-flight, walk or wavelength decision).
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _equal_fraction(a, b, rel):
    return float(np.mean(np.all(np.abs(a - b) <= rel * np.maximum(1.0, np.abs(b)), axis=-1)))


def test_cornell_full_size_image(pe, device, oracle):
    scene, cam, st = scenes().cornell_box(256, 256, 64, 8, seed=0)
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    r = device.render(cam, st, pe.RenderTargets(beauty=film), 0, 64)
    assert r.completed and r.samples_traced == 256 * 256 * 64
    ref = oracle.RefScene(scene)
    mean_ref, cnt_ref = ref.render(cam, st, 0, 64)
    assert np.array_equal(film.count, cnt_ref)
    img = film.resolve()
    err = pe.rel_mse(img, mean_ref)
    same = _equal_fraction(img, mean_ref, 1e-5)
    assert err <= 1e-6, (err, same)
    assert same >= 0.99, same


def test_knot_full_size_primary_hits(pe, device, oracle):
    scene, cam, st = scenes().torus_knot_scene(1920, 1080, 256, 12)
    scene.build_accelerator()
    assert scene.info.triangles == 4096 * 128 * 2 + 4
    device.set_scene(scene)
    ref = oracle.RefScene(scene)
    for sample in (0, 5):
        rs, rp, rt = ref.trace_primary(cam, st, sample)
        # the binary tree in the reference's visiting order: every id and distance bit-exact
        ms, mp, mt = device.trace_primary(cam, st, sample, ordered=True)
        assert np.array_equal(ms, rs) and np.array_equal(mp, rp)
        assert np.array_equal(mt.view(np.uint32), rt.view(np.uint32))
        # the 4-wide tree the render kernels trace: every distance bit-exact, ids equal except at
        # ties (two triangles at the identical distance: a ray through a shared edge)
        ms, mp, mt = device.trace_primary(cam, st, sample)
        same = (ms == rs) & (mp == rp)
        ties = ~same & (mp >= 0) & (rp >= 0)
        assert np.array_equal(mt.view(np.uint32), rt.view(np.uint32))
        assert np.array_equal(~same, ties), np.count_nonzero(~same & ~ties)
        assert np.count_nonzero(ties) <= 1e-4 * ms.size, np.count_nonzero(ties)


def test_media_full_size_image(pe, device, oracle):
    scene, cam, st = scenes().media_scene(1280, 720, 512, 24)
    scene.build_accelerator()
    assert scene.info.lights >= 2000 and scene.info.light_sampler_mode == 2
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, 2)
    ref = oracle.RefScene(scene)
    mean_ref, cnt_ref = ref.render(cam, st, 0, 2)
    assert np.array_equal(film.count, cnt_ref)
    img = film.resolve()
    err = pe.rel_mse(img, mean_ref)
    same = _equal_fraction(img, mean_ref, 1e-4)
    assert err <= 3e-3, (err, same)
    assert same >= 0.99, same
