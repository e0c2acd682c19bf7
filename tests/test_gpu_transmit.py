"""Shadow rays through thin-walled glass and cutout surfaces (shadowTransmittance,
path_tracer.cpp:172-202) and closest-hit rays through cutouts (passesCutout, :161-167), against
the reference engine's CPU path at equal spp.  These paths use no transcendental functions
beyond the plain Cornell ones, so the bound is the plain one."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _scene(pe, with_glass=True, with_cutout=True):
    scene, cam, st = scenes().cornell_box(64, 64, 16, 8, seed=9)
    S = scenes()
    if with_glass:
        pane = pe.Dielectric(1.5, tint=(0.9, 0.8, 0.6))
        pane.set_thin_walled(True)
        p, i = S._quad((1.0, 0.2, 1.2), (1.0, 3.6, 1.2), (4.4, 3.6, 1.2), (4.4, 0.2, 1.2))
        scene.add_shape(pe.TriangleMesh(p, None, None, i, pane))
    if with_cutout:
        leaf = pe.DisneyMaterial((0.2, 0.6, 0.2), 0.0, 0.5, 0.5)
        leaf.set_opacity(0.4)
        p, i = S._quad((1.5, 4.5, 1.0), (4.0, 4.5, 1.0), (4.0, 4.5, 4.0), (1.5, 4.5, 4.0))
        scene.add_shape(pe.TriangleMesh(p, None, None, i, leaf))
    return scene, cam, st


@pytest.mark.parametrize("glass,cutout", [(True, False), (False, True), (True, True)])
def test_transmitting_surfaces_match_reference(pe, device, oracle, glass, cutout):
    scene, cam, st = _scene(pe, glass, cutout)
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, 16)
    mean_ref, cnt_ref = oracle.RefScene(scene).render(cam, st, 0, 16)
    assert np.array_equal(film.count, cnt_ref)
    img = film.resolve()
    err = pe.rel_mse(img, mean_ref)
    same = np.mean(np.all(np.abs(img - mean_ref) <= 1e-5 * np.maximum(1.0, np.abs(mean_ref)), axis=-1))
    assert err < 1e-4, (err, same)
    assert same > 0.95, (err, same)
