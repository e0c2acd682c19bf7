"""Thin-lens (round and polygonal aperture) and orthographic cameras on the CUDA path against the
reference's own camera classes driving its CPU path, on the Cornell box at equal spp.

Tolerance: the aperture warps call cosf / sinf (CUDA and glibc differ by an ulp or two), so a
camera ray can leave the reference's by an ulp and graze an edge differently; images agree to
relMSE ≤ 1e-4 with ≥ 99 % of the pixels equal to 1e-4 relative, and without bias."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["thin-lens", "thin-lens-pentagon", "orthographic"])
def test_camera_renders_match_reference(pe, device, oracle, kind):
    S = importlib.import_module("photon_engine_b200.scenes")
    scene, _, st = S.cornell_box(64, 64, 8, 8, seed=0)
    eye, tgt, up = (2.78, 2.73, -8.0), (2.78, 2.73, 0.0), (0.0, 1.0, 0.0)
    if kind == "thin-lens":
        cam = pe.ThinLensCamera(eye, tgt, up, 39.0, 1.0, 0.25, 9.0)
    elif kind == "thin-lens-pentagon":
        cam = pe.ThinLensCamera(eye, tgt, up, 39.0, 1.0, 0.25, 9.0, 5, 20.0)
    else:
        cam = pe.OrthographicCamera(eye, tgt, up, 6.0, 1.0)
    scene.build_accelerator()
    device.set_scene(scene)
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, 8)
    ref, cnt = oracle.RefScene(scene).render(cam, st, 0, 8)
    assert np.array_equal(film.count, cnt)
    img = film.resolve()
    err = pe.rel_mse(img, ref)
    same = np.mean(np.all(np.abs(img - ref) <= 1e-4 * np.maximum(1.0, np.abs(ref)), axis=-1))
    bias = float(img.mean() / ref.mean() - 1.0)
    assert err < 1e-4 and same > 0.99 and abs(bias) < 1e-3, (err, same, bias)
