"""The device's tuning knobs (pe_tuning) change how fast a film is made, never the film: every
4-wide closest-hit traversal variant (stack in local memory, first 8 / 16 entries in shared
memory, top 4 / 8 entries in registers, a 64-register cap) visits the same nodes in the same
order, the any-hit variants answer the same, the shading register budgets and tail thresholds
run the same code, so their films are bit-identical; the binary tree may resolve a
bit-identical distance tie to the other triangle of a shared edge, and so may the walk with
postponed leaf tests, so their films are compared at the equal-spp bar.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tuning_knobs_leave_the_film_unchanged(pe, device):
    S = importlib.import_module("photon_engine_b200.scenes")
    scene, cam, st = S.torus_knot_scene(160, 90, 4, 8, nu=256, nv=16, env_size=(128, 64))
    scene.build_accelerator()
    device.set_scene(scene)

    def film(**kw):
        device.set_tuning(**kw)
        f = pe.Film(st.width, st.height)
        device.render(cam, st, pe.RenderTargets(beauty=f), 0, 4)
        return f

    try:
        base = film(closest_traversal=1, shade_budget=1, any_traversal=0)
        for mode in (2, 3, 4, 5, 6, 7, 8):
            f = film(closest_traversal=mode, shade_budget=1, any_traversal=0)
            assert np.array_equal(f.sum, base.sum) and np.array_equal(f.count, base.count), mode
        for kw in ({"any_traversal": 1}, {"any_traversal": 2}, {"shade_budget": 0}, {"shade_budget": 2}, {"tail_paths": 1024}, {"tail_paths": 0}):
            args = {"closest_traversal": 1, "shade_budget": 1, "any_traversal": 0, **kw}
            f = film(**args)
            assert np.array_equal(f.sum, base.sum), kw
        # postponed leaf tests (mode 9) visit leaves in another order: ties may go the other way
        spec = film(closest_traversal=9, shade_budget=1, any_traversal=0)
        assert np.array_equal(spec.count, base.count)
        assert pe.rel_mse(spec.resolve(), base.resolve()) <= 1e-4
        binary = film(closest_traversal=0, shade_budget=1, any_traversal=0)
        assert np.array_equal(binary.count, base.count)
        assert pe.rel_mse(binary.resolve(), base.resolve()) <= 1e-4
    finally:
        device.set_tuning()


def test_wave_slots_leave_the_film_unchanged(pe, device):
    """Paths in flight per wave (pe_tuning::wave_slots): 3.7M paths through 1M slots regenerate
    paths in freed slots, through 4M slots they all start at once; the film is the same."""
    S = importlib.import_module("photon_engine_b200.scenes")
    scene, cam, st = S.torus_knot_scene(640, 360, 16, 8, nu=256, nv=16, env_size=(128, 64))
    scene.build_accelerator()
    device.set_scene(scene)

    def film(slots):
        device.set_tuning(wave_slots=slots)
        assert device.tuning()["wave_slots"] == slots
        f = pe.Film(st.width, st.height)
        device.render(cam, st, pe.RenderTargets(beauty=f), 0, 16)
        return f

    try:
        small, large = film(1 << 20), film(1 << 22)
        assert np.array_equal(small.count, large.count)
        assert np.array_equal(small.sum, large.sum) and np.array_equal(small.sum_sq, large.sum_sq)
        with pytest.raises(Exception):
            device.set_tuning(wave_slots=1 << 24)
    finally:
        device.set_tuning()
