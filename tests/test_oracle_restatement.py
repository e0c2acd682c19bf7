"""The C restatement of the hot path (oracle/pe_oracle.c) pinned to the reference: against the
golden fixtures generated from the reference's own CPU path (tests/golden/make_golden.py) and,
where the compiled reference is present, against it directly.  CPU only."""
import importlib
import pathlib

import numpy as np
import pytest

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def orc():
    import oracle
    if not oracle.restatement_available():
        pytest.skip("oracle/_ref/libpe_oracle.so not built (make -C oracle restatement)")
    return oracle


def test_restated_sobol_matches_golden_vectors(orc):
    g = np.load(GOLDEN / "sobol_vectors.npz")
    for si, seed in enumerate(g["seeds"]):
        for k in range(0, len(g["px"]), 7):
            v = orc.restated_sobol(int(seed), int(g["px"][k]), int(g["py"][k]), int(g["index"][k]), 12)
            assert np.array_equal(v.view(np.uint32), g["values"][si, k].view(np.uint32)), (seed, k)


def test_compiled_reference_matches_golden_vectors(oracle):
    g = np.load(GOLDEN / "sobol_vectors.npz")
    for si, seed in enumerate(g["seeds"]):
        v = oracle.sobol(int(seed), g["px"], g["py"], g["index"], 12)
        assert np.array_equal(v.view(np.uint32), g["values"][si].view(np.uint32))


def cornell(w, h, spp=8):
    sc = importlib.import_module("photon_engine_b200.scenes")
    return sc.cornell_box(w, h, spp, 8, seed=0)


def test_restated_primary_hits_match_golden(orc):
    g = np.load(GOLDEN / "cornell_32.npz")
    scene, cam, st = cornell(32, 32)
    shape, prim, t = orc.Restatement(scene).trace_primary(cam, st, 0)
    assert np.array_equal(shape, g["shape"]) and np.array_equal(prim, g["prim"])
    assert np.array_equal(t.view(np.uint32), g["t"].view(np.uint32))


def test_restated_image_matches_golden(pe, orc):
    g = np.load(GOLDEN / "cornell_32.npz")
    scene, cam, st = cornell(32, 32)
    mean = orc.Restatement(scene).render(cam, st, 0, 8)
    assert pe.rel_mse(mean, g["mean"]) < 1e-10
    assert np.array_equal(mean.view(np.uint32), g["mean"].view(np.uint32))


def test_restatement_matches_reference_at_64(pe, orc, oracle):
    scene, cam, st = cornell(64, 64, 4)
    res = orc.Restatement(scene)
    ref = oracle.RefScene(scene)
    for s in (0, 3):
        a = res.trace_primary(cam, st, s)
        b = ref.trace_primary(cam, st, s)
        assert all(np.array_equal(x, y) for x, y in zip(a[:2], b[:2]))
    mine = res.render(cam, st, 0, 4)
    theirs, _ = ref.render(cam, st, 0, 4)
    assert pe.rel_mse(mine, theirs) < 1e-10
