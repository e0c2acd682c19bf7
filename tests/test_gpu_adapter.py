"""The drop-in itself: the C++ RenderDevice adapter (photon-engine_b200/adapter/cuda_render_device.cpp)
compiled against the reference engine's headers and linked with the reference engine and
libphoton_cuda.so (oracle/Makefile target `adapter`), driven by the reference's own
RenderSession::begin / advance (src/engine/render_session.cpp:17-101) on a reference Scene.

Its films must be the films the Python mirror of the API renders through the same library for the
same scene, camera and samples: equal sample counts, and sums equal up to the float rounding of
adding the session's batches in a different grouping (relMSE ≤ 1e-10).
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


@pytest.fixture(scope="module")
def adapter_oracle(oracle):
    if not oracle.adapter_available():
        pytest.fail("oracle/_ref/libpe_adapter.so missing: build it with `make -C oracle adapter`")
    return oracle


def _mirror(pe, device, scene, cam, st, spp, aovs=False):
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    targets = pe.RenderTargets(beauty=film, aovs=pe.AovFilms(st.width, st.height) if aovs else None)
    r = device.render(cam, st, targets, 0, spp)
    assert r.completed
    return film, targets.aovs


def test_adapter_reports_features_and_renders_the_mirror_film(pe, device, adapter_oracle):
    scene, cam, st = scenes().torus_knot_scene(96, 54, 16, 8, nu=192, nv=12, env_size=(128, 64))
    film, aov = _mirror(pe, device, scene, cam, st, 16, aovs=True)
    ref = adapter_oracle.RefScene(scene, fast="adapter")
    mean, cnt, alb, done, feats = ref.session_cuda(cam, st, 16, batch=5, aovs=True)
    assert feats == 7, "features(): aovs, lightPasses and adaptiveSampling"
    assert done == 16
    assert np.array_equal(cnt, film.count)
    assert pe.rel_mse(mean, film.resolve()) <= 1e-10
    assert pe.rel_mse(alb, aov.albedo.resolve()) <= 1e-10


def test_adapter_incremental_updates_match_a_rebuilt_mirror(pe, device, adapter_oracle):
    scene, cam, st = scenes().torus_knot_scene(64, 36, 8, 6, nu=128, nv=8, env_size=(64, 32))
    ref = adapter_oracle.RefScene(scene, fast="adapter")
    ref.session_cuda(cam, st, 4, batch=4)
    # SceneUpdateKind::Materials: a Disney base colour; SceneUpdateKind::Lights: the softbox
    mats = scene.materials()
    k = next(i for i, m in enumerate(mats) if m.struct.type == pe._capi.PE_MAT_DISNEY)
    ref.session_cuda_update(1, ref.mat_index[id(mats[k])], (0.9, 0.1, 0.2))
    ref.session_cuda_update(2, 0, (3.0, 6.0, 9.0))
    mean, cnt, _, _, _ = ref.session_cuda(cam, st, 8, batch=8)
    mats[k].struct.base_color = pe._capi.f3((0.9, 0.1, 0.2))
    area = next(obj for kind, obj in scene.ops if kind == "area")
    area.radiance = (3.0, 6.0, 9.0)
    film, _ = _mirror(pe, device, scene, cam, st, 8)
    assert np.array_equal(cnt, film.count)
    assert pe.rel_mse(mean, film.resolve()) <= 1e-10


def test_adapter_adaptive_session_converges(pe, device, adapter_oracle):
    scene, cam, st = scenes().cornell_box(48, 48, 64, 6, seed=12345)
    st.noise_threshold = 0.05
    st.min_adaptive_samples = 8
    scene.build_accelerator()
    ref = adapter_oracle.RefScene(scene, fast="adapter")
    mean, cnt, _, done, _ = ref.session_cuda(cam, st, 64, batch=8, adaptive=True)
    assert np.isfinite(mean).all() and mean.mean() > 0.0
    assert cnt.min() >= 8 and cnt.max() <= 64
    assert cnt.mean() < 64, "no pixel stopped early"


def test_adapter_carries_instances_and_their_transforms(pe, device, adapter_oracle):
    """MeshInstances through the adapter (one BLAS per mesh), then SceneUpdateKind::Transforms with
    the instances placed anew in the reference scene: the adapter refits, the mirror refits."""
    H = importlib.import_module("test_instances")
    scene, cam, st = H.instanced_cornell(pe, 48, 48, 8, 6)
    st.seed = 12345  # Renderer::renderSamples' Sobol seed, which the session uses
    film, _ = _mirror(pe, device, scene, cam, st, 8)
    ref = adapter_oracle.RefScene(scene, fast="adapter")
    mean, cnt, _, done, _ = ref.session_cuda(cam, st, 8, batch=3)
    assert done == 8 and np.array_equal(cnt, film.count)
    assert pe.rel_mse(mean, film.resolve()) <= 1e-10
    n = scene.shape_count()
    moved = [H.rot_y(1.1, (2.2, 0.8, 2.0), 1.0), H.rot_y(0.2, (3.2, 2.0, 3.0), 0.7)]
    for k, m in enumerate(moved):
        ref.move_instance(n - 2 + k, m)
    ref.session_cuda_update(3)
    mean, cnt, _, _, _ = ref.session_cuda(cam, st, 8, batch=8)
    inst = [o for kind, o in scene.ops if kind == "instance"]
    for o, m in zip(inst, moved):
        o.local_to_world, o.world_to_local = m, None
    assert device.update_scene(scene, pe.SceneUpdateKind.Transforms)
    film2 = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film2), 0, 8)
    assert np.array_equal(cnt, film2.count)
    assert pe.rel_mse(mean, film2.resolve()) <= 1e-10
