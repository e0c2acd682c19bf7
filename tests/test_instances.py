"""Mesh instancing on the host side (MeshInstance, src/geometry/mesh_instance.h; Scene::addShape,
src/scene/scene.cpp:23-41): the C ABI's BLAS / instance / refit entry points, their limits and
errors, the scene counts an instanced scene reports, and the reference engine tracing the same
instances (oracle/_ref).  No GPU: the device half is tests/test_gpu_instances.py.
"""
import ctypes as C
import importlib

import numpy as np
import pytest


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def cube(pe, material, size=0.5):
    """12 triangles: one BLAS leaf (at most 16 triangles keep the reference's BVH on one leaf)."""
    p = np.array([[x, y, z] for x in (-size, size) for y in (-size, size) for z in (-size, size)], np.float32)
    f = np.array([[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1],
                  [2, 3, 7], [2, 7, 6], [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]], np.uint32)
    return pe.TriangleMesh(p, None, None, f, material)


def rot_y(a, t=(0.0, 0.0, 0.0), s=1.0):
    c, n = np.cos(a), np.sin(a)
    m = np.array([[c * s, 0, n * s, t[0]], [0, s, 0, t[1]], [-n * s, 0, c * s, t[2]], [0, 0, 0, 1]], np.float32)
    return m


def instanced_cornell(pe, w=48, h=48, spp=4, depth=6, emissive=False):
    scene, cam, st = scenes().cornell_box(w, h, spp, depth, seed=5)
    red = pe.DisneyMaterial((0.8, 0.2, 0.1), 0.0, 0.4)
    mesh = cube(pe, red)
    scene.add_shape(pe.MeshInstance(mesh, rot_y(0.5, (1.5, 0.6, 1.6), 1.2)))
    scene.add_shape(pe.MeshInstance(mesh, rot_y(-0.3, (3.8, 0.5, 2.8), 0.9), pe.Mirror((0.9, 0.9, 0.9))))
    if emissive:
        glow = pe.Lambertian((0.0, 0.0, 0.0))
        glow.struct.emission = pe._capi.f3((4.0, 3.0, 2.0))
        scene.add_shape(pe.MeshInstance(cube(pe, glow, 0.2), rot_y(0.0, (2.8, 2.5, 3.5))))
    return scene, cam, st


def test_instances_count_their_mesh_once(pe):
    scene, cam, st = instanced_cornell(pe)
    scene.build_accelerator()
    base, _, _ = scenes().cornell_box(48, 48, 4, 6, seed=5)
    base.build_accelerator()
    assert scene.info.triangles == base.info.triangles + 12, "one BLAS of 12 triangles for both instances"
    assert scene.info.lights == base.info.lights


def test_emissive_instance_gives_a_light_per_triangle(pe):
    scene, _, _ = instanced_cornell(pe, emissive=True)
    scene.build_accelerator()
    base, _, _ = instanced_cornell(pe)
    base.build_accelerator()
    assert scene.info.lights == base.info.lights + 12


def test_instance_abi_rejects_bad_input(pe):
    lib = pe._capi.load()
    s = lib.pe_scene_create()
    try:
        p = np.zeros((3, 3), np.float32)
        p[1, 0] = p[2, 1] = 1.0
        idx = np.array([0, 1, 2], np.uint32)
        eye = np.eye(4, dtype=np.float32)
        f = pe._capi.fptr
        assert lib.pe_scene_add_blas(s, f(p), 3, None, None, pe._capi.uptr(idx), 1) == 0
        bad = np.array([0, 1, 7], np.uint32)
        assert lib.pe_scene_add_blas(s, f(p), 3, None, None, pe._capi.uptr(bad), 1) == -pe._capi.PE_ERR_INVALID
        m = lib.pe_scene_add_material(s, C.byref(pe.Lambertian((0.5, 0.5, 0.5)).struct))
        assert lib.pe_scene_add_instance(s, 5, f(eye), f(eye), m) != pe._capi.PE_OK, "no such BLAS"
        assert lib.pe_scene_add_instance(s, 0, f(eye), f(eye), 99) != pe._capi.PE_OK, "no such material"
        for _ in range(1024):
            assert lib.pe_scene_add_instance(s, 0, f(eye), f(eye), m) == pe._capi.PE_OK
        assert lib.pe_scene_build(s) == pe._capi.PE_ERR_LIMIT, "at most 1023 instances a scene"
        assert b"1023" in lib.pe_last_error()
    finally:
        lib.pe_scene_destroy(s)


def test_set_transform_edits_instances_only(pe):
    scene, cam, st = instanced_cornell(pe, emissive=True)
    scene.build_accelerator()
    lib = pe._capi.load()
    f = pe._capi.fptr
    eye = np.eye(4, dtype=np.float32)
    n = scene.shape_count()
    assert lib.pe_scene_set_instance_transform(scene.handle, 0, f(eye), f(eye)) == pe._capi.PE_ERR_INVALID
    assert lib.pe_scene_set_instance_transform(scene.handle, n - 3, f(eye), f(eye)) == pe._capi.PE_OK
    assert lib.pe_scene_set_instance_transform(scene.handle, n - 1, f(eye), f(eye)) == pe._capi.PE_ERR_LIMIT, \
        "an emissive instance moves its lights: rebuild"
    assert lib.pe_scene_refit(scene.handle) == pe._capi.PE_OK
    assert not scene.sync_transforms(), "the emissive instance refuses a refit"


def test_reference_traces_the_instances(pe, oracle):
    scene, cam, st = instanced_cornell(pe)
    scene.build_accelerator()
    ref = oracle.RefScene(scene)
    shape, prim, t = ref.trace_primary(cam, st, 0)
    n = scene.shape_count()
    assert (shape == n - 2).sum() > 20 and (shape == n - 1).sum() > 20
    assert prim[shape >= n - 2].max() < 12


def test_reference_moved_instance_traces_as_a_scene_built_moved(pe, oracle):
    """The oracle's move_instance (a new MeshInstance in the old slot) is the scene built with the
    new matrix: the reference side of the Transforms update tests."""
    scene, cam, st = instanced_cornell(pe)
    scene.build_accelerator()
    ref = oracle.RefScene(scene)
    n = scene.shape_count()
    moved = rot_y(1.1, (2.2, 0.8, 2.0), 1.0)
    ref.move_instance(n - 2, moved)
    _, inst = [(k, o) for k, o in scene.ops if k == "instance"][0]
    inst.local_to_world = moved
    inst.world_to_local = None
    scene.build_accelerator()
    fresh = oracle.RefScene(scene)
    a, b = ref.trace_primary(cam, st, 1), fresh.trace_primary(cam, st, 1)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    with pytest.raises(ValueError):
        ref.move_instance(0, moved)


def moving_cornell(pe, w=48, h=48, spp=4, depth=6, seed=12345):
    """The instanced Cornell box with its red cube moving (translation, a half turn and a scale
    change over the shutter) and the mirror cube static."""
    scene, cam, st = instanced_cornell(pe, w, h, spp, depth)
    st.seed = seed
    inst = [o for k, o in scene.ops if k == "instance"]
    inst[0].set_motion_transform(rot_y(2.0, (2.2, 1.3, 2.0), 0.8))
    return scene, cam, st


def test_moving_instance_bounds_match_reference(pe, oracle):
    """MeshInstance::recomputeBounds over the shutter: the union of five interpolated poses
    (interpolateTransform: decomposeTRS, SLERP in double, composeTRS) bit for bit."""
    scene, cam, st = moving_cornell(pe)
    scene.build_accelerator()
    lib = pe._capi.load()
    ref = oracle.RefScene(scene)
    kind, tris, bounds = oracle.scene_shapes(ref)
    out = np.empty(6, np.float32)
    for i in range(scene.shape_count()):
        assert lib.pe_scene_shape_bounds(scene.handle, i, pe._capi.fptr(out)) == pe._capi.PE_OK
        assert np.array_equal(out, bounds[i]), (i, out, bounds[i])
    n = scene.shape_count()
    static = rot_y(0.5, (1.5, 0.6, 1.6), 1.2)
    lo = bounds[n - 2][:3]
    assert (lo < static[:3, 3] - 0.5).any(), "the moving cube's box spans the shutter"


def test_moving_instance_refuses_a_refit(pe):
    scene, cam, st = moving_cornell(pe)
    scene.build_accelerator()
    lib = pe._capi.load()
    eye = np.eye(4, dtype=np.float32)
    n = scene.shape_count()
    f = pe._capi.fptr
    assert lib.pe_scene_set_instance_transform(scene.handle, n - 2, f(eye), f(eye)) == pe._capi.PE_ERR_LIMIT
    assert lib.pe_scene_set_instance_motion(scene.handle, 0, f(eye), None) == pe._capi.PE_ERR_INVALID
