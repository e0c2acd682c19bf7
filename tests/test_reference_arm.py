"""The reference arm of bench.py runs the reference's own CPU path only: its scene comes from the
plain-numpy workload description, and the process maps no product library."""
import json
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle  # noqa: E402

needs_ref = pytest.mark.skipif(not oracle.available(fast=True), reason="oracle/_ref not built")


@needs_ref
def test_reference_arm_loads_no_product_library():
    code = f"""
import json, sys
sys.path.insert(0, {str(ROOT)!r})
import bench
sys.path.insert(0, {str(ROOT / 'oracle')!r})
import oracle
desc = bench.workload_description(48, 27, 128, 8, (64, 32))
ref = oracle.ref_scene_from_description(desc, fast=True)
cam = oracle.DescCamera(desc["camera"], fast=True)
st = oracle.DescSettings(desc["settings"])
mean, cnt = oracle.render_stock(ref, cam, st, 0, 1, 2)
print(json.dumps({{"libs": bench.loaded_libraries(), "mean": float(mean.mean()), "count": int(cnt.sum()),
                  "config": bench.workload_config(desc)}}))
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    res = json.loads(out.stdout.strip().splitlines()[-1])
    assert res["libs"], "the reference library should be mapped"
    assert all(lib.startswith("oracle/_ref/") for lib in res["libs"]), res["libs"]
    assert res["count"] == 48 * 27 and res["mean"] > 0.0
    assert res["config"]["triangles"] == 2 * 128 * 8 + 4


@needs_ref
def test_description_scene_equals_product_scene_on_the_reference():
    """The reference scene built from the description renders the same film as the reference
    scene replayed from the product Scene built from that description."""
    import pe_pkg
    pe = pe_pkg.load()
    from photon_engine_b200 import scenegen, scenes
    desc = scenegen.torus_knot(40, 24, 4, 6, nu=96, nv=8, env_size=(64, 32))
    scene, cam, st = scenes.from_description(desc)
    a = oracle.RefScene(scene)
    mean_a, cnt_a = a.render(cam, st, 3, 2, threads=2, seeded=False)
    b = oracle.ref_scene_from_description(desc)
    mean_b, cnt_b = oracle.render_stock(b, oracle.DescCamera(desc["camera"]), oracle.DescSettings(desc["settings"]),
                                        3, 2, threads=2)
    assert np.array_equal(cnt_a, cnt_b)
    assert np.array_equal(mean_a, mean_b)


def test_material_defaults_agree():
    """The oracle's description defaults are the ABI's pe_material_defaults."""
    import ctypes as C
    import pe_pkg
    pe = pe_pkg.load()
    if not oracle.available():
        pytest.skip("oracle/_ref not built")
    lib = pe._capi.load()
    ref = oracle._load()
    for t in range(4):
        a, b = pe._capi.pe_material(), pe._capi.pe_material()
        lib.pe_material_defaults(t, C.byref(a))
        ref.ref_material_defaults(t, C.byref(b))
        assert bytes(a) == bytes(b), t
