"""Adaptive sampling on the CUDA path (RenderSettings::adaptiveSampling) against the reference
engine's Renderer::renderSamples on the same film, scene and Owen-Sobol indices (seed 12345):

* a pixel whose 3×3 neighbourhood is below the noise threshold skips the batch, once the film
  holds minAdaptiveSamples (renderer.cpp:442-467);
* within a batch, a pixel stops after a sample index that is a multiple of 8 (at least
  minAdaptiveSamples, before the batch's end) once its relative error (Film::relativeError,
  film.cpp:100-109) is below the threshold (renderer.cpp:498-500).

Each pixel takes the same samples as in the reference, and the device film adds them in the
same order to the same accumulated sums, so the per-pixel sample counts and the samples traced
must be equal, and the images agree to the beauty film's parity tolerance (relMSE ≤ 1e-6).
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _adaptive(st, threshold, min_spp):
    st.seed = 12345
    st.adaptive_sampling = True
    st.noise_threshold = threshold
    st.min_adaptive_samples = min_spp
    return st


@pytest.mark.parametrize("batches", [[(0, 48)], [(0, 16), (16, 24), (40, 24)]])
def test_adaptive_counts_and_film_match_reference(pe, device, oracle, batches):
    scene, cam, st = scenes().cornell_box(48, 48, 8, 6, seed=0)
    _adaptive(st, 0.08, 16)
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    ref = oracle.RefScene(scene)
    rfilm = oracle.RefFilm(st.width, st.height)
    for first, count in batches:
        r = device.render(cam, st, pe.RenderTargets(beauty=film), first, count)
        traced = ref.render_into(rfilm, cam, st, first, count)
        mean, cnt = rfilm.mean_and_counts()
        assert np.array_equal(film.count, cnt), (first, count, int(np.sum(film.count != cnt)))
        assert r.samples_traced == traced, (first, count, r.samples_traced, traced)
        assert pe.rel_mse(film.resolve(), mean) < 1e-6
    # some pixels stopped early, some went on to the end
    total = batches[-1][0] + batches[-1][1]
    assert film.count.min() < total and film.count.max() == total, (film.count.min(), film.count.max())


def test_session_converges(pe, device):
    """RenderSession with adaptive sampling ends once a batch traces nothing
    (test_render_session.cpp:176-195)."""
    scene, cam, st = scenes().cornell_box(32, 32, 8, 6, seed=0)
    # the pixels beside the ceiling light keep a relative error above 0.05 well past 4096 spp
    _adaptive(st, 0.2, 8)
    scene.build_accelerator()
    device.set_scene(scene)
    sess = pe.RenderSession(device)
    sess.begin(cam, st, pe.SessionConfig(target_spp=4096))
    while sess.advance():
        pass
    assert not sess.warnings
    assert sess.converged()
    assert sess.samples < 4096
    assert sess.average_samples() < 1000.0


def test_adaptive_off_takes_every_sample(pe, device):
    scene, cam, st = scenes().cornell_box(32, 32, 8, 6, seed=0)
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    r = device.render(cam, st, pe.RenderTargets(beauty=film), 0, 24)
    assert int(film.count.min()) == 24 and r.samples_traced == 24 * 32 * 32
