"""SD-tree path guiding (RenderSettings.path_guiding; the reference's GuidingField and its use in
PathTracer::Li and Renderer::renderSamples) on the CUDA path.

Guided renders are not bit-reproducible, on either side: splats reach the trees through float
atomics in whatever order the threads run, and the sampling decisions follow the trees.  The
checks are therefore statistical: the training schedule (refinements at 2, 4, 8, 16 and 32
samples, a new field from sample 0 or on a new scene), an unbiased image against a converged
plain render, the reference's own guided render agreeing in mean and error, and the error at
equal spp against the plain render.

Metric: relMSE (mean of (x − r)² / (r² + 0.01), the reference's compare script) on images
scaled so the converged mean is 0.18, averaged over independent Sobol seeds.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _render(pe, device, cam, st, first, count, batch=None):
    film = pe.Film(st.width, st.height)
    batch = batch or count
    for s0 in range(first, first + count, batch):
        device.render(cam, st, pe.RenderTargets(beauty=film), s0, min(batch, first + count - s0))
    return film.resolve()


@pytest.fixture()
def room(pe, device):
    scene, cam, st = scenes().room_scene(96, 54, 32, 8, knot_res=(128, 16), env_size=(256, 128))
    scene.build_accelerator()
    device.set_scene(scene)
    yield scene, cam, st
    st.path_guiding = False
    device.set_guiding(0)


@pytest.fixture()
def cornell(pe, device):
    scene, cam, st = scenes().cornell_box(64, 64, 64, 8, seed=0)
    scene.build_accelerator()
    device.set_scene(scene)
    yield scene, cam, st
    st.path_guiding = False
    device.set_guiding(0)


def test_training_schedule(pe, device, cornell):
    scene, cam, st = cornell
    st.path_guiding = True
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, 1)
    i = device.sdtree_info()
    assert (i.refinements, i.ready, i.samples) == (0, 0, 1)
    device.render(cam, st, pe.RenderTargets(beauty=film), 1, 7)     # 1→2, 2→4, 4→8
    i = device.sdtree_info()
    assert (i.refinements, i.samples) == (3, 8) and i.ready and i.spatial_leaves >= 8 and i.energy > 0
    device.render(cam, st, pe.RenderTargets(beauty=film), 8, 40)    # 8→16, 16→32, frozen after
    i = device.sdtree_info()
    assert (i.refinements, i.samples) == (5, 32) and i.ready
    # the box's records (most paths find the light) split the spatial tree past its 8 initial leaves
    assert i.spatial_leaves > 8, i.spatial_leaves
    assert i.quad_nodes > i.spatial_leaves, i.quad_nodes
    assert np.all(film.count == 48) and np.all(np.isfinite(film.resolve()))
    device.render(cam, st, pe.RenderTargets(beauty=film), 48, 16)   # frozen: no refinement
    assert device.sdtree_info().refinements == 5
    # a render from sample 0 starts a new field
    device.render(cam, st, pe.RenderTargets(beauty=pe.Film(st.width, st.height)), 0, 4)
    assert device.sdtree_info().refinements == 2
    # so does a new scene
    device.set_scene(scene)
    device.render(cam, st, pe.RenderTargets(beauty=pe.Film(st.width, st.height)), 4, 2)
    assert device.sdtree_info().refinements == 1
    # turning the setting off drops the field
    st.path_guiding = False
    device.render(cam, st, pe.RenderTargets(beauty=pe.Film(st.width, st.height)), 0, 1)
    assert device.sdtree_info().refinements == 0


def test_guided_room_unbiased_and_as_good_as_reference(pe, device, room, oracle):
    """The indirect-lit room at 128 spp from sample 0 (32 of them training samples): the guided
    image is unbiased, and its error matches the reference's own guided CPU render of the same
    view.  Neither beats the plain render at this spp on this small frame: the spatial tree
    keeps its 8 initial leaves (few paths reach the window), and half the samples at each
    guided vertex follow a field averaged over a 5 m × 1.5 m × 4 m cell."""
    scene, cam, st = room
    ref = _render(pe, device, cam, st, 1 << 20, 8192, batch=1024)
    k = 0.18 / float(ref.mean())

    def err(img):
        return pe.rel_mse(img * k, ref * k)

    spp = 128
    plain, guided = [], []
    for i in range(12):
        st.seed = 1000 + i
        st.path_guiding = False
        plain.append(_render(pe, device, cam, st, 0, spp))
        st.path_guiding = True
        guided.append(_render(pe, device, cam, st, 0, spp))
        assert device.sdtree_info().refinements == 5
    st.path_guiding = False
    # the reference: a new Renderer per call, so each sample range trains a field of its own
    R = oracle.RefScene(scene)
    theirs = [R.render_guided(cam, st, 1000 * i, spp)[0] for i in range(6)]
    e_plain = float(np.mean([err(x) for x in plain]))
    e_guided = float(np.mean([err(x) for x in guided]))
    e_theirs = float(np.mean([err(x) for x in theirs]))
    print(f"room relMSE at {spp} spp: plain {e_plain:.4g}, SD-tree guided {e_guided:.4g}, "
          f"reference guided {e_theirs:.4g}")
    bias = float(np.mean(guided) / ref.mean() - 1.0)
    assert abs(bias) < 0.03, bias
    assert e_guided < 1.3 * e_theirs, (e_guided, e_theirs)


def test_guided_cornell_agrees_with_reference(pe, device, oracle):
    """The reference's guided render of the same Cornell box (its CPU path, 64 spp from sample
    0): both images estimate the same converged image, with errors of the same size."""
    scene, cam, st = scenes().cornell_box(48, 48, 64, 8, seed=0)
    scene.build_accelerator()
    device.set_scene(scene)
    try:
        ref = _render(pe, device, cam, st, 1 << 20, 8192, batch=1024)
        st.path_guiding = True
        mine = _render(pe, device, cam, st, 0, 64)
        assert device.sdtree_info().refinements == 5
    finally:
        st.path_guiding = False
        device.set_guiding(0)
    theirs, cnt = oracle.RefScene(scene).render_guided(cam, st, 0, 64)
    assert np.all(cnt == 64)
    k = 0.18 / float(ref.mean())
    e_mine = pe.rel_mse(mine * k, ref * k)
    e_theirs = pe.rel_mse(theirs * k, ref * k)
    print(f"Cornell 64 spp guided relMSE: CUDA {e_mine:.4g}, reference CPU {e_theirs:.4g}")
    assert abs(float(mine.mean() / ref.mean()) - 1.0) < 0.02
    assert abs(float(theirs.mean() / ref.mean()) - 1.0) < 0.02
    assert e_mine < 2.0 * e_theirs, (e_mine, e_theirs)


def test_adaptive_and_guided_together(pe, device, oracle):
    """Adaptive sampling with the SD-tree on in one render (Renderer::renderSamples runs both,
    renderer.cpp:413-526): the field trains on the pixels still rendering, pixels stop at the
    8-sample checks; the reference's own adaptive guided render of the same view is the
    comparison.  Both are unbiased against a converged plain render, take a similar number of
    samples, and reach a similar error."""
    scene, cam, st = scenes().cornell_box(48, 48, 64, 8, seed=0)
    scene.build_accelerator()
    device.set_scene(scene)
    try:
        ref = _render(pe, device, cam, st, 1 << 20, 8192, batch=1024)
        st.path_guiding = True
        st.adaptive_sampling = True
        st.noise_threshold = 0.05
        st.min_adaptive_samples = 8
        film = pe.Film(st.width, st.height)
        device.render(cam, st, pe.RenderTargets(beauty=film), 0, 64)
        info = device.sdtree_info()
        mine, cnt = film.resolve(), film.count
    finally:
        st.path_guiding = False
        st.adaptive_sampling = False
        device.set_guiding(0)
    assert info.refinements == 5 and info.ready
    assert cnt.min() >= 8 and cnt.max() <= 64 and cnt.mean() < 64, "some pixels stop early"
    st.path_guiding = True
    st.adaptive_sampling = True
    theirs, tcnt = oracle.RefScene(scene).render_guided(cam, st, 0, 64)
    st.path_guiding = False
    st.adaptive_sampling = False
    assert tcnt.min() >= 8 and tcnt.mean() < 64
    assert abs(cnt.mean() / tcnt.mean() - 1.0) < 0.15, (cnt.mean(), tcnt.mean())
    k = 0.18 / float(ref.mean())
    e_mine = pe.rel_mse(mine * k, ref * k)
    e_theirs = pe.rel_mse(theirs * k, ref * k)
    assert abs(float(mine.mean() / ref.mean()) - 1.0) < 0.03
    assert e_mine < 1.5 * e_theirs, (e_mine, e_theirs)
