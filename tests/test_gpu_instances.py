"""Mesh instancing on the CUDA path (MeshInstance, src/geometry/mesh_instance.cpp:104-133) against the
reference engine's CPU path: one BLAS per mesh, one top-level primitive per instance, rays carried
into the instance's space by its world-to-local matrix and the hit record carried back by
transformHitToWorld (mesh_instance.cpp:56-101).

Tolerances:
  * instances of at most 16 triangles (one BLAS leaf, where the reference's own traversal is
    sound): primary-hit shape, triangle and distance bit-exact on the binary tree in the
    reference's order, distances bit-exact on the 4-wide tree; images at equal spp relMSE ≤ 1e-4
    with ≥ 99 % of pixels equal to 1e-4 relative;
  * a large instanced mesh (1024 triangles) against the same mesh flattened into world space in the
    reference's scene (the reference drops hits behind an instance of more than 16 triangles, a
    defect of its shared traversal stack, tests/test_project.py): the instance's floats differ from
    the flattened mesh's by a rounding, so ≥ 99.5 % of primary hits name the same shape with
    distances within 1e-4 relative, and images at 64 spp relMSE ≤ 2e-3;
  * SceneUpdateKind::Transforms (a refit of the top-level tree) against a rebuilt scene: primary
    distances bit-exact, films relMSE ≤ 1e-6 (the refitted tree may meet a tie in another order).
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def helpers():
    return importlib.import_module("test_instances")


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def check_hits_bit_exact(device, ref, scene, cam, st, samples=(0, 2)):
    for s in samples:
        rs, rp, rt = ref.trace_primary(cam, st, s)
        ms, mp, mt = device.trace_primary(cam, st, s, ordered=True)
        assert np.array_equal(ms, rs) and np.array_equal(mp, rp)
        assert np.array_equal(mt.view(np.uint32), rt.view(np.uint32))
        _, _, wt = device.trace_primary(cam, st, s)
        assert np.array_equal(wt.view(np.uint32), rt.view(np.uint32))


def image_close(pe, img, ref, tol=1e-4, share=0.99):
    err = pe.rel_mse(img, ref)
    same = float(np.mean(np.all(np.abs(img - ref) <= 1e-4 * np.maximum(1.0, np.abs(ref)), axis=-1)))
    assert err <= tol, (err, same)
    assert same >= share, same


def render(pe, device, scene, cam, st, spp):
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, spp)
    return film


def test_small_instances_hit_bit_exact(pe, device, oracle):
    scene, cam, st = helpers().instanced_cornell(pe, 64, 64)
    scene.build_accelerator()
    device.set_scene(scene)
    ref = oracle.RefScene(scene)
    check_hits_bit_exact(device, ref, scene, cam, st)
    shape, _, _ = device.trace_primary(cam, st, 0)
    n = scene.shape_count()
    assert (shape == n - 1).sum() > 20 and (shape == n - 2).sum() > 20


def test_explicit_inverse_is_used_as_given(pe, device, oracle):
    """world_to_local given by the caller (Transform(m, inverse)) reaches both sides as given."""
    scene, cam, st = helpers().instanced_cornell(pe, 64, 64)
    for kind, obj in scene.ops:
        if kind == "instance":
            obj.world_to_local = np.linalg.inv(obj.local_to_world.astype(np.float64)).astype(np.float32)
    scene.build_accelerator()
    device.set_scene(scene)
    check_hits_bit_exact(device, oracle.RefScene(scene), scene, cam, st, samples=(1,))


def test_instance_images_match_reference_at_equal_spp(pe, device, oracle):
    scene, cam, st = helpers().instanced_cornell(pe, 64, 64, 8, 8, emissive=True)
    scene.build_accelerator()
    device.set_scene(scene)
    film = render(pe, device, scene, cam, st, 8)
    mean_ref, cnt_ref = oracle.RefScene(scene).render(cam, st, 0, 8)
    assert np.array_equal(film.count, cnt_ref)
    image_close(pe, film.resolve(), mean_ref)


def knot_pair(pe):
    """The Cornell box with a 1024-triangle knot: as a MeshInstance (rotated, scaled, moved) and as
    the same mesh with its vertices carried to world space."""
    S = scenes()
    pos, quads = S.torus_knot_mesh(64, 8, seed=1)
    q = quads.reshape(-1, 4)
    tri = np.concatenate([q[:, [0, 1, 2]], q[:, [0, 2, 3]]]).astype(np.uint32)
    mat = pe.DisneyMaterial((0.7, 0.3, 0.2), 0.0, 0.3)
    m = helpers().rot_y(0.6, (2.7, 1.4, 2.6), 0.45)
    out = []
    for flat in (False, True):
        scene, cam, st = S.cornell_box(96, 96, 64, 6, seed=9)
        p = pos.astype(np.float32)
        if flat:
            w = (p.astype(np.float64) @ m[:3, :3].T.astype(np.float64) + m[:3, 3]).astype(np.float32)
            scene.add_shape(pe.TriangleMesh(w, None, None, tri, mat))
        else:
            scene.add_shape(pe.MeshInstance(pe.TriangleMesh(p, None, None, tri, mat), m))
        scene.build_accelerator()
        out.append((scene, cam, st))
    return out


def test_large_instance_matches_the_flattened_mesh(pe, device, oracle):
    (inst, cam, st), (flat, _, _) = knot_pair(pe)
    device.set_scene(inst)
    ms, _, mt = device.trace_primary(cam, st, 0)
    rs, _, rt = oracle.RefScene(flat).trace_primary(cam, st, 0)
    n = inst.shape_count()
    assert (rs == n - 1).sum() > 300, "the knot covers the frame's middle"
    agree = ms == rs
    assert agree.mean() >= 0.995, agree.mean()
    both = agree & (rs >= 0)
    assert np.allclose(mt[both], rt[both], rtol=1e-4)
    film = render(pe, device, inst, cam, st, 64)
    mean_ref, _ = oracle.RefScene(flat).render(cam, st, 0, 64)
    assert pe.rel_mse(film.resolve(), mean_ref) <= 2e-3


def test_transforms_update_refits_like_a_rebuild(pe, device, oracle):
    H = helpers()
    scene, cam, st = H.instanced_cornell(pe, 64, 64, 8, 6)
    scene.build_accelerator()
    device.set_scene(scene)
    render(pe, device, scene, cam, st, 2)
    inst = [o for k, o in scene.ops if k == "instance"]
    inst[0].local_to_world = H.rot_y(1.1, (2.2, 0.8, 2.0), 1.0)
    inst[1].local_to_world = H.rot_y(0.2, (3.2, 2.0, 3.0), 0.7)
    for o in inst:
        o.world_to_local = None
    assert device.update_scene(scene, pe.SceneUpdateKind.Transforms), "refit refused"
    refit_hits = device.trace_primary(cam, st, 1)
    refit = render(pe, device, scene, cam, st, 8)
    scene.build_accelerator()
    device.set_scene(scene)
    fresh_hits = device.trace_primary(cam, st, 1)
    fresh = render(pe, device, scene, cam, st, 8)
    assert np.array_equal(refit_hits[2].view(np.uint32), fresh_hits[2].view(np.uint32))
    assert np.array_equal(refit.count, fresh.count)
    assert pe.rel_mse(refit.resolve(), fresh.resolve()) <= 1e-6
    rs, _, rt = oracle.RefScene(scene).trace_primary(cam, st, 1)
    assert np.array_equal(refit_hits[2].view(np.uint32), rt.view(np.uint32))


def test_instanced_grid_keeps_one_mesh(pe, device):
    """A 10×10 grid of one 1024-triangle mesh: one BLAS on the device, not 100 copies."""
    S = scenes()
    pos, quads = S.torus_knot_mesh(64, 8, seed=1)
    q = quads.reshape(-1, 4)
    tri = np.concatenate([q[:, [0, 1, 2]], q[:, [0, 2, 3]]]).astype(np.uint32)
    mesh = pe.TriangleMesh(pos.astype(np.float32), None, None, tri, pe.DisneyMaterial((0.5, 0.6, 0.7), 1.0, 0.2))
    scene, cam, st = S.cornell_box(64, 64, 4, 6, seed=2)
    for i in range(10):
        for j in range(10):
            scene.add_shape(pe.MeshInstance(mesh, helpers().rot_y(0.3 * i, (0.5 + 0.45 * i, 0.3, 0.5 + 0.45 * j), 0.08)))
    scene.build_accelerator()
    assert scene.info.triangles == 36 + 1024
    device.set_scene(scene)
    film = render(pe, device, scene, cam, st, 4)
    assert np.isfinite(film.resolve()).all()
