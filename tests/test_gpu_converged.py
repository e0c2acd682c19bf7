"""Converged images against the reference: 16384-spp crops of each workload rendered by the
reference engine's CPU path (fixtures from tests/golden/make_converged.py, the windows listed
there) and by the device through pe_device_render_region with the same samples
[0, 16384) of the same Sobol seed.  Gate: relMSE (mean over pixels and channels of
(x − ref)² / (ref² + 0.01)) ≤ 1e-3 on every window, and the sample counts equal.
"""
import importlib.util
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def _generator():
    spec = importlib.util.spec_from_file_location("make_converged", GOLDEN / "make_converged.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def rel_mse(x, ref):
    return float(np.mean((x.astype(np.float64) - ref) ** 2 / (ref.astype(np.float64) ** 2 + 0.01)))


@pytest.mark.parametrize("name", ["cornell", "knot", "media", "room"])
def test_converged_windows_match_reference(pe, device, name):
    z = np.load(GOLDEN / f"converged_{name}.npz")
    gen = _generator()
    scene, cam, st = gen.build(name)
    st.seed = int(z["seed"])
    scene.build_accelerator()
    device.set_scene(scene)
    spp = int(z["spp"])
    film = pe.Film(st.width, st.height)
    errs = []
    for k, rect in enumerate(z["rects"]):
        x0, y0, w, h = (int(v) for v in rect)
        device.render_region(cam, st, film, (x0, y0, w, h), 0, spp)
        win = (slice(y0, y0 + h), slice(x0, x0 + w))
        assert np.array_equal(film.count[win], z["count"][k])
        mean = film.sum[win] / np.maximum(film.count[win], 1)[..., None]
        errs.append(rel_mse(mean, z["mean"][k]))
    assert max(errs) <= 1e-3, errs
