"""Generates the golden fixtures of this folder by running the reference engine's own CPU path
(oracle/_ref/libphoton_ref.so, built from the reference sources by oracle/Makefile).

    python tests/golden/make_golden.py

sobol_vectors.npz   Owen-scrambled Sobol values: 500 (pixel, sample index) pairs x 12 2-D
                    dimensions for three seeds, the inputs drawn like the reference's
                    MatchesReferenceDefinitionBitExact test (pixels in [0, 4096), the first 64
                    indices 0..63, the rest random 31-bit).
cornell_32.npz      the 36-triangle Cornell box at 32x32, seed 0: primary-hit shape/prim/t for
                    sample 0 and the mean image of samples [0, 8), depth 8.
"""
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import importlib  # noqa: E402

import oracle  # noqa: E402
import pe_pkg  # noqa: E402


def main():
    pe_pkg.load()
    out = pathlib.Path(__file__).resolve().parent
    rng = np.random.default_rng(77)
    n = 500
    px = rng.integers(0, 4096, n).astype(np.int32)
    py = rng.integers(0, 4096, n).astype(np.int32)
    idx = np.where(np.arange(n) < 64, np.arange(n), rng.integers(0, 2**31 - 1, n)).astype(np.int32)
    seeds = np.array([0, 12345, 0x1234567890ABCDEF], np.uint64)
    vals = np.stack([oracle.sobol(int(s), px, py, idx, 12) for s in seeds])
    np.savez_compressed(out / "sobol_vectors.npz", px=px, py=py, index=idx, seeds=seeds, values=vals)

    sc = importlib.import_module("photon_engine_b200.scenes")
    scene, cam, st = sc.cornell_box(32, 32, 8, 8, seed=0)
    ref = oracle.RefScene(scene)
    shape, prim, t = ref.trace_primary(cam, st, 0)
    mean, cnt = ref.render(cam, st, 0, 8)
    np.savez_compressed(out / "cornell_32.npz", shape=shape, prim=prim, t=t, mean=mean, count=cnt)
    print("wrote", out / "sobol_vectors.npz", out / "cornell_32.npz")


if __name__ == "__main__":
    main()
