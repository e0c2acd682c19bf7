"""pe_scene_set_material (the host half of RenderDevice::updateScene with
SceneUpdateKind::Materials, render_device.h:77-79): parameter edits are taken in place; a change
of type, emission or a scene-level switch (media, shadow transmission) asks for a rebuild."""
import numpy as np


def test_material_edits_and_rejections(pe):
    lib = pe._capi.load()
    s = lib.pe_scene_create()
    try:
        d = pe.DisneyMaterial((0.5, 0.5, 0.5), 0.0, 0.5)
        idx = lib.pe_scene_add_material(s, d.struct)
        assert idx == 0
        tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
        assert lib.pe_scene_add_mesh(s, pe._capi.fptr(tri), 3, None, None,
                                     pe._capi.uptr(np.array([0, 1, 2], np.uint32)), 1, idx) == 0
        assert lib.pe_scene_build(s) == 0
        e = pe.DisneyMaterial((0.9, 0.1, 0.1), 1.0, 0.2)       # new colour, metal, roughness
        assert lib.pe_scene_set_material(s, idx, e.struct) == pe._capi.PE_OK
        assert lib.pe_scene_set_material(s, idx, pe.Lambertian((0.5, 0.5, 0.5)).struct) != pe._capi.PE_OK
        glow = pe.DisneyMaterial((0.5, 0.5, 0.5), 0.0, 0.5)
        glow.struct.emission[0] = 3.0
        assert lib.pe_scene_set_material(s, idx, glow.struct) != pe._capi.PE_OK
        cut = pe.DisneyMaterial((0.5, 0.5, 0.5), 0.0, 0.5)
        cut.set_opacity(0.5)                                    # makes it a shadow transmitter
        assert lib.pe_scene_set_material(s, idx, cut.struct) != pe._capi.PE_OK
        assert lib.pe_scene_set_material(s, 1, e.struct) != pe._capi.PE_OK
    finally:
        lib.pe_scene_destroy(s)
