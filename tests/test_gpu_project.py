"""A .photon project rendered on the device: this repository's own project fixture
(tests/golden/studio.photon: transformed groups of meshes, spheres under a scaling transform,
Disney / glass / mirror / Lambert materials, an area light, the ground quad, the procedural studio
sky, a Gaussian pixel filter) loaded by photon-engine_b200/project.py.

* against the reference's CPU path on the same loaded scene and samples: relMSE ≤ 1e-4 with
  ≥ 99 % of pixels equal to 1e-4 relative, as the other equal-spp parity renders;
* end to end against the reference's own loadProject + buildRenderScene of the same file (the
  loader builds the reference's scene bit for bit: mesh nodes as MeshInstances, tests/test_project.py),
  the same bar at 16 spp.
"""
import importlib
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PROJECT = pathlib.Path(__file__).resolve().parent / "golden" / "studio.photon"


def test_project_renders_as_the_reference(pe, device, oracle):
    proj = importlib.import_module("photon_engine_b200.project")
    scene, cam, st = proj.load_project(PROJECT, 96, 72, 16)
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, 16)
    img = film.resolve()
    mean_ref, cnt = oracle.RefScene(scene).render(cam, st, 0, 16)
    assert np.array_equal(film.count, cnt)
    err = pe.rel_mse(img, mean_ref)
    same = float(np.mean(np.all(np.abs(img - mean_ref) <= 1e-4 * np.maximum(1.0, np.abs(mean_ref)), axis=-1)))
    assert err <= 1e-4 and same >= 0.99, (err, same)


def test_project_end_to_end_against_the_reference_loader(pe, device, oracle):
    proj = importlib.import_module("photon_engine_b200.project")
    scene, cam, st = proj.load_project(PROJECT, 96, 72, 16)
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, 16)
    ref, rcam, *_ = oracle.load_project(PROJECT, 96, 72)
    mean_ref, cnt = oracle.RefScene.render(ref, rcam, st, 0, 16)
    assert np.array_equal(film.count, cnt)
    img = film.resolve()
    err = pe.rel_mse(img, mean_ref)
    same = float(np.mean(np.all(np.abs(img - mean_ref) <= 1e-4 * np.maximum(1.0, np.abs(mean_ref)), axis=-1)))
    assert err <= 1e-4 and same >= 0.99, (err, same)
