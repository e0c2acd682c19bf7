"""RenderSettings::shadowQuality > 1 on the CUDA path against the reference engine's CPU path:
several NEE samples per vertex (path_tracer.cpp:631-698: the sample loop, each term weighted
by powerHeuristic(n, lightPdf, 1, bsdfPdf) / n, emission hits by powerHeuristic(1, ·, n, ·)),
as many contact-AO rays, four times as many shadow-catcher rays.  Such waves shade with their
shadow rays traced in the shading kernel, each sample's term added in the sample loop's order.

Tolerance: images at equal spp relMSE ≤ 1e-4 with ≥ 99 % of pixels equal to 1e-4 relative.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _compare(pe, device, oracle, scene, cam, st, spp):
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, spp)
    mean_ref, cnt_ref = oracle.RefScene(scene).render(cam, st, 0, spp)
    assert np.array_equal(film.count, cnt_ref)
    img = film.resolve()
    err = pe.rel_mse(img, mean_ref)
    same = float(np.mean(np.all(np.abs(img - mean_ref) <= 1e-4 * np.maximum(1.0, np.abs(mean_ref)), axis=-1)))
    assert err <= 1e-4 and same >= 0.99, (err, same)
    return img


@pytest.mark.parametrize("quality", [2, 4])
def test_cornell_shadow_quality_matches_reference(pe, device, oracle, quality):
    scene, cam, st = scenes().cornell_box(64, 64, 8, 8, seed=0)
    st.shadow_quality = quality
    img = _compare(pe, device, oracle, scene, cam, st, 8)
    # several shadow rays a vertex lower the noise against quality 1 at the same spp
    st.shadow_quality = 1
    one = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=one), 0, 8)
    assert abs(img.mean() / one.resolve().mean() - 1.0) < 0.05


def test_knot_shadow_quality_with_sky_sun_and_ao(pe, device, oracle):
    scene, cam, st = scenes().torus_knot_scene(96, 54, 8, 8, nu=192, nv=12, env_size=(128, 64))
    st.shadow_quality = 3
    st.ao_strength = 0.5
    _compare(pe, device, oracle, scene, cam, st, 4)


def test_server_refuses_shadow_quality_above_one(pe, device):
    scene, cam, st = scenes().cornell_box(32, 32, 4, 4, seed=0)
    scene.build_accelerator()
    st.shadow_quality = 2
    srv = pe.RenderServer(device, 1 << 30)
    try:
        sid = srv.add_scene(scene)
        with pytest.raises(pe._capi.PhotonError):
            srv.submit(sid, cam, st, 4)
    finally:
        srv.close()
