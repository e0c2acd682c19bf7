"""The tile render that allocates no device memory (pe_device_render_tile_noalloc).

It exists for hosts that may not call cudaMalloc while they render — a viewport or plugin
inside another application that owns the GPU memory budget and hands out buffers from its own
pool, or a render thread that must not enter the driver's allocator mid-frame.  The film is
memory the caller owns; the path state is the library's fixed scratch array.  Its output must
equal, bit for bit, what the allocating entry point (pe_device_render) adds for the same pixels
and samples: the same paths, summed per pixel in the same sample order.
This file sorts last so a run that stops at the first failure has run every other test.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _cornell(pe, w, h):
    return _scenes().cornell_box(w, h, 4, 8, seed=0)


def _media(pe, w, h):
    # dispersive glass, a scattering and an absorbing volume, a subsurface slab, 2000 LED triangles
    return _scenes().media_scene(w, h, 4, 16, sphere_res=(48, 24), cyl_res=(48, 8), slab_res=6)


def _textured(pe, w, h):
    scene, cam, st = _scenes().cornell_box(w, h, 4, 6, seed=0)
    rng = np.random.default_rng(5)
    m = pe.DisneyMaterial((0.8, 0.8, 0.8), 0.0, 0.4)
    m.set_albedo_image(np.kron(rng.uniform(0.05, 0.95, (4, 4, 3)).astype(np.float32), np.ones((8, 8, 1), np.float32)))
    m.set_texture_mapping(True)
    pos, nrm, idx = _scenes().uv_sphere((2.78, 1.2, 2.2), 0.9, 32, 16)
    scene.add_shape(pe.TriangleMesh(pos, nrm, None, idx, m))
    return scene, cam, st


def _film_buffers(st):
    import torch
    torch.cuda.set_device(0)
    s = torch.zeros((st.height, st.width, 3), dtype=torch.float32, device="cuda")
    c = torch.zeros((st.height, st.width), dtype=torch.int32, device="cuda")
    q = torch.zeros((st.height, st.width), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    return s, c, q


@pytest.mark.parametrize("make", [_cornell, _media, _textured], ids=["cornell", "media", "textured"])
def test_tile_matches_allocating_entry_point_over_two_calls(pe, device, make):
    import torch

    scene, cam, st = make(pe, 96, 64)
    scene.build_accelerator()
    device.set_scene(scene)
    ref = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=ref), 0, 4)

    s, c, q = _film_buffers(st)
    x0, y0, w, h = 16, 8, 64, 40
    # two calls in a row: the second finds the first call's scratch contents and must not care
    device.render_tile_noalloc(cam, st, x0, y0, w, h, 0, 2, s.data_ptr(), c.data_ptr(), q.data_ptr())
    device.render_tile_noalloc(cam, st, x0, y0, w, h, 2, 2, s.data_ptr(), c.data_ptr(), q.data_ptr())
    device.synchronize()
    torch.cuda.synchronize()
    sn, cn, qn = s.cpu().numpy(), c.cpu().numpy().astype(np.uint32), q.cpu().numpy()

    tile = (slice(y0, y0 + h), slice(x0, x0 + w))
    assert np.array_equal(cn[tile], ref.count[tile])
    assert np.array_equal(sn[tile], ref.sum[tile])
    assert np.array_equal(qn[tile], ref.sum_sq[tile])
    outside = np.ones(cn.shape, bool)
    outside[tile] = False
    assert not cn[outside].any() and not sn[outside].any()


def test_tile_above_maximum_is_rejected(pe, device):
    import torch

    scene, cam, st = _cornell(pe, 256, 256)
    scene.build_accelerator()
    device.set_scene(scene)
    buf = torch.zeros(256 * 256 * 3, dtype=torch.float32, device="cuda")
    with pytest.raises(pe._capi.PhotonError, match="exceeds the maximum of 32768 pixels"):
        device.render_tile_noalloc(cam, st, 0, 0, 256, 256, 0, 1, buf.data_ptr(), buf.data_ptr(), buf.data_ptr())


def test_tile_rejects_films_it_cannot_write(pe, device):
    """A host pointer and a buffer smaller than the film are refused before any kernel runs."""
    import torch

    scene, cam, st = _cornell(pe, 64, 64)
    scene.build_accelerator()
    device.set_scene(scene)
    s, c, q = _film_buffers(st)
    host = np.zeros((64, 64, 3), np.float32)
    with pytest.raises(pe._capi.PhotonError, match="device"):
        device.render_tile_noalloc(cam, st, 0, 0, 32, 32, 0, 1, host.ctypes.data, c.data_ptr(), q.data_ptr())
    # a buffer of its own (torch's caching allocator would hand out a slice of a larger block)
    from cuda.bindings import runtime as rt
    err, short = rt.cudaMalloc(400)
    assert err == rt.cudaError_t.cudaSuccess
    try:
        with pytest.raises(pe._capi.PhotonError, match="the film needs"):
            device.render_tile_noalloc(cam, st, 0, 0, 32, 32, 0, 1, s.data_ptr(), c.data_ptr(), int(short))
    finally:
        rt.cudaFree(short)
    # the device still renders afterwards
    device.render_tile_noalloc(cam, st, 0, 0, 32, 32, 0, 1, s.data_ptr(), c.data_ptr(), q.data_ptr())
    device.synchronize()
    assert int(c.sum().item()) == 32 * 32


def test_tile_rejects_guided_devices_and_mipmapped_scenes(pe, device):
    scene, cam, st = _cornell(pe, 64, 64)
    scene.build_accelerator()
    device.set_scene(scene)
    s, c, q = _film_buffers(st)
    lib = pe._capi.load()
    pe._capi.check(lib.pe_device_set_guiding(device.handle, 1, 1, 3e-3))
    try:
        with pytest.raises(pe._capi.PhotonError, match="guided"):
            device.render_tile_noalloc(cam, st, 0, 0, 32, 32, 0, 1, s.data_ptr(), c.data_ptr(), q.data_ptr())
    finally:
        pe._capi.check(lib.pe_device_set_guiding(device.handle, 0, 0, 0.0))
    scene, cam, st = _cornell(pe, 64, 64)
    m = pe.DisneyMaterial((0.8, 0.8, 0.8), 0.0, 0.4)
    m.set_albedo_image(np.full((16, 16, 3), 0.5, np.float32), mipmaps=True)
    pos, nrm, idx = _scenes().uv_sphere((2.78, 1.2, 2.2), 0.9, 16, 8)
    scene.add_shape(pe.TriangleMesh(pos, nrm, None, idx, m))
    scene.build_accelerator()
    device.set_scene(scene)
    with pytest.raises(pe._capi.PhotonError, match="mipmapped"):
        device.render_tile_noalloc(cam, st, 0, 0, 32, 32, 0, 1, s.data_ptr(), c.data_ptr(), q.data_ptr())
