"""RenderDevice::updateScene with SceneUpdateKind::Materials on the CUDA device
(render_device.h:77-79): edited material parameters reach the device without a rebuild, and the
frame equals a frame of a freshly built scene with the edited materials, bit for bit."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_material_update_equals_rebuild(pe, device):
    S = importlib.import_module("photon_engine_b200.scenes")
    scene, cam, st = S.cornell_box(48, 48, 8, 6, seed=0)
    m = pe.DisneyMaterial((0.3, 0.5, 0.7), 0.0, 0.6, 0.5)
    p, n, i = S.uv_sphere((2.8, 1.2, 2.8), 1.0, 32, 16)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, m))
    scene.build_accelerator()
    device.set_scene(scene)
    before = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=before), 0, 4)
    # edit in place: colour, metalness, roughness, clearcoat
    m.struct.base_color[:] = (0.9, 0.2, 0.1)
    m.struct.metallic = 1.0
    m.struct.roughness = 0.25
    m.struct.clearcoat = 0.7
    assert device.update_scene(scene, pe.SceneUpdateKind.Materials) is True
    updated = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=updated), 0, 4)
    assert pe.rel_mse(updated.resolve(), before.resolve()) > 1e-4
    # the same scene built from scratch
    scene.build_accelerator()
    device.set_scene(scene)
    rebuilt = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=rebuilt), 0, 4)
    assert np.array_equal(updated.sum, rebuilt.sum) and np.array_equal(updated.count, rebuilt.count)
    # a change of type falls back to a rebuild
    scene.ops[-1][1].material = pe.Lambertian((0.5, 0.5, 0.5))
    assert device.update_scene(scene, pe.SceneUpdateKind.Materials) is False


def test_light_update_equals_rebuild(pe, device):
    """SceneUpdateKind::Lights: a new AreaLight radiance reaches the device (lights, the quad's
    emission, the light sampler) without a rebuild; the frame equals a rebuilt scene's."""
    S = importlib.import_module("photon_engine_b200.scenes")
    scene, cam, st = S.cornell_box(48, 48, 8, 6, seed=0)
    key = pe.AreaLight((1.0, 4.5, 1.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), (6.0, 6.0, 6.0))
    scene.add_light(key)
    scene.build_accelerator()
    device.set_scene(scene)
    before = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=before), 0, 4)
    key.radiance = (20.0, 9.0, 3.0)
    assert device.update_scene(scene, pe.SceneUpdateKind.Lights) is True
    updated = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=updated), 0, 4)
    assert pe.rel_mse(updated.resolve(), before.resolve()) > 1e-4
    scene.build_accelerator()
    device.set_scene(scene)
    rebuilt = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=rebuilt), 0, 4)
    assert np.array_equal(updated.sum, rebuilt.sum) and np.array_equal(updated.count, rebuilt.count)
