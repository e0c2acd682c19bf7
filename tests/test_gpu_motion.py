"""Motion blur on the CUDA path (RenderSettings::motionBlur) against the reference engine's CPU
path: each camera sample draws a shutter time (Sobol dimension 2, renderer.cpp:152-153); the
camera mixes its two poses at that time (Camera::generateRay(u, v, lens, time), camera.h:58-90);
a moving MeshInstance meets the ray under interpolateTransform (quat.cpp: translation and scale
linear, rotation by SLERP in double precision) for the closest hit, the hit record, shadow rays
and every other ray of the path.

Tolerance: images at equal spp relMSE ≤ 1e-4 with ≥ 99 % of pixels equal to 1e-4 relative, the
bar of the other equal-spp parity renders (the SLERP's sines are CUDA's on the device, glibc's on
the host, within an ulp of each other in double before the float rounding).
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def helpers():
    return importlib.import_module("test_instances")


def render(pe, device, scene, cam, st, spp):
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, spp)
    return film


def image_close(pe, img, ref, tol=1e-4, share=0.99):
    err = pe.rel_mse(img, ref)
    same = float(np.mean(np.all(np.abs(img - ref) <= 1e-4 * np.maximum(1.0, np.abs(ref)), axis=-1)))
    assert err <= tol and same >= share, (err, same)


def test_moving_instance_matches_reference(pe, device, oracle):
    scene, cam, st = helpers().moving_cornell(pe, 64, 64, 8, 6)
    st.motion_blur = True
    film = render(pe, device, scene, cam, st, 8)
    mean_ref, cnt = oracle.RefScene(scene).render(cam, st, 0, 8)
    assert np.array_equal(film.count, cnt)
    image_close(pe, film.resolve(), mean_ref)
    # the blur is there: the same scene without motion blur differs
    st.motion_blur = False
    still = render(pe, device, scene, cam, st, 8)
    assert pe.rel_mse(still.resolve(), film.resolve()) > 1e-3


def test_without_motion_blur_a_moving_instance_stays_at_its_first_pose(pe, device):
    H = helpers()
    scene, cam, st = H.moving_cornell(pe, 48, 48, 4, 6)
    moving = render(pe, device, scene, cam, st, 4)
    still, _, _ = H.instanced_cornell(pe, 48, 48, 4, 6)
    film = render(pe, device, still, cam, st, 4)
    assert np.array_equal(moving.count, film.count)
    assert np.array_equal(moving.sum, film.sum)


@pytest.mark.parametrize("kind", ["perspective", "thin_lens"])
def test_camera_shutter_end_matches_reference(pe, device, oracle, kind):
    scene, cam, st = helpers().instanced_cornell(pe, 64, 64, 8, 6)
    st.seed = 12345
    st.motion_blur = True
    if kind == "perspective":
        cam = pe.PerspectiveCamera((2.78, 2.73, -8.0), (2.78, 2.73, 2.8), (0, 1, 0), 37.0, 1.0)
        end = pe.PerspectiveCamera((3.3, 2.9, -7.6), (2.6, 2.6, 2.8), (0, 1, 0), 40.0, 1.0)
    else:
        cam = pe.ThinLensCamera((2.78, 2.73, -8.0), (2.78, 2.73, 2.8), (0, 1, 0), 37.0, 1.0, 0.08, 10.0, 6, 15.0)
        end = pe.ThinLensCamera((3.3, 2.9, -7.6), (2.6, 2.6, 2.8), (0, 1, 0), 40.0, 1.0, 0.15, 9.0, 6, 15.0)
    cam.set_shutter_end(end)
    film = render(pe, device, scene, cam, st, 8)
    mean_ref, cnt = oracle.RefScene(scene).render(cam, st, 0, 8)
    assert np.array_equal(film.count, cnt)
    image_close(pe, film.resolve(), mean_ref)
