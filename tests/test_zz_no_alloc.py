"""The tile render that allocates no device memory (pe_device_render_tile_noalloc).

It exists for hosts that may not call cudaMalloc while they render — a viewport or plugin
inside another application that owns the GPU memory budget and hands out buffers from its own
pool, or a render thread that must not enter the driver's allocator mid-frame.  The film is
memory the caller owns; the path state is the library's fixed scratch array.  Its output must
equal what the allocating entry point (pe_device_render) adds for the same pixels and samples.
This file sorts last so a run that stops at the first failure has run every other test.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene(pe, device, width, height):
    sc = importlib.import_module("photon_engine_b200.scenes")
    scene, cam, st = sc.cornell_box(width, height, 4, 8, seed=0)
    scene.build_accelerator()
    device.set_scene(scene)
    return cam, st


def test_tile_matches_allocating_entry_point_over_two_calls(pe, device):
    import torch

    cam, st = _scene(pe, device, 96, 64)
    ref = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=ref), 0, 4)

    torch.cuda.set_device(0)
    s = torch.zeros((st.height, st.width, 3), dtype=torch.float32, device="cuda")
    c = torch.zeros((st.height, st.width), dtype=torch.int32, device="cuda")
    q = torch.zeros((st.height, st.width), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    x0, y0, w, h = 16, 8, 64, 40
    # two calls in a row: the second finds the first call's scratch contents and must not care
    device.render_tile_noalloc(cam, st, x0, y0, w, h, 0, 2, s.data_ptr(), c.data_ptr(), q.data_ptr())
    device.render_tile_noalloc(cam, st, x0, y0, w, h, 2, 2, s.data_ptr(), c.data_ptr(), q.data_ptr())
    torch.cuda.synchronize()
    sn, cn, qn = s.cpu().numpy(), c.cpu().numpy().astype(np.uint32), q.cpu().numpy()

    tile = (slice(y0, y0 + h), slice(x0, x0 + w))
    assert np.array_equal(cn[tile], ref.count[tile])
    # same paths, same per-pixel summation order: equal to the tolerance the parity tests use
    np.testing.assert_allclose(sn[tile], ref.sum[tile], rtol=1e-6, atol=0.0)
    np.testing.assert_allclose(qn[tile], ref.sum_sq[tile], rtol=1e-6, atol=0.0)
    outside = np.ones(cn.shape, bool)
    outside[tile] = False
    assert not cn[outside].any() and not sn[outside].any()


def test_tile_above_maximum_is_rejected(pe, device):
    import dataclasses

    import torch

    cam, st = _scene(pe, device, 256, 256)
    big = dataclasses.replace(st)
    buf = torch.zeros(256 * 256 * 3, dtype=torch.float32, device="cuda")
    with pytest.raises(pe._capi.PhotonError, match="exceeds the maximum of 32768 pixels"):
        device.render_tile_noalloc(cam, big, 0, 0, 256, 256, 0, 1, buf.data_ptr(), buf.data_ptr(), buf.data_ptr())
