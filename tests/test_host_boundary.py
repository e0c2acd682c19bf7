"""Host side of the boundary against the reference (no GPU): camera description, scene
flattening (lights, light-sampler mode) and input validation."""
import ctypes as C
import importlib

import numpy as np
import pytest


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


@pytest.mark.parametrize("args", [((2.78, 2.73, -8.0), (2.78, 2.73, 0.0), (0.0, 1.0, 0.0), 39.3, 1.0),
                                  ((0.0, 4.5, -10.5), (0.0, 1.6, 0.0), (0.0, 1.0, 0.0), 40.0, 16 / 9),
                                  ((1.0, 2.0, 3.0), (-4.0, 0.5, 2.0), (0.0, 0.0, 1.0), 65.0, 1.25)])
def test_camera_description_bit_exact(pe, oracle, args):
    mine = pe.PerspectiveCamera(*args).describe_gpu()
    ref = oracle.camera_perspective(*args, pe._capi.pe_camera())
    for f in ("position", "lower_left", "horizontal", "vertical", "u", "v", "forward"):
        assert list(getattr(mine, f)) == list(getattr(ref, f)), f


def test_cornell_lights_and_sampler_mode_match_reference(pe, oracle):
    scene, cam, st = scenes().cornell_box()
    scene.build_accelerator()
    ref = oracle.RefScene(scene)
    assert scene.info.lights == ref.light_count() == 2
    assert scene.info.light_sampler_mode == ref.light_mode() == 1
    assert scene.info.triangles == 36


def test_area_light_adds_two_triangles_and_one_light(pe, oracle):
    scene, cam, st = scenes().cornell_box()
    scene.add_light(pe.AreaLight((1, 5, 1), (1, 0, 0), (0, 0, 1), (5, 5, 5)))
    scene.build_accelerator()
    ref = oracle.RefScene(scene)
    assert scene.info.triangles == 38
    assert scene.info.lights == ref.light_count() == 3


def test_mesh_index_out_of_range_is_rejected(pe):
    scene = pe.Scene()
    mat = pe.Lambertian((0.5, 0.5, 0.5))
    scene.add_shape(pe.TriangleMesh(np.zeros((3, 3), np.float32), None, None, np.array([[0, 1, 5]], np.uint32), mat))
    with pytest.raises(pe._capi.PhotonError, match="out of range"):
        scene.build_accelerator()
