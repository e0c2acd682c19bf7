"""The SD-tree's directional quadtree (pe_sdtree.h, the code the shading kernels run) against the
reference's DirectionalTree (src/integrators/path_guiding.cpp:80-222) on the host: the same
splats in two training passes with a refinement between them must give the same tree, so the
same pdf for every direction and the same (direction, pdf) for every sample, bit for bit.  Both
sides are compiled without FMA contraction and call the same libm functions."""
import ctypes as C

import numpy as np
import pytest


def _fp(a):
    return np.ascontiguousarray(a, np.float32).ctypes.data_as(C.POINTER(C.c_float))


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def _splats(rng, n, centres, spread):
    """Directions around a few centres (plus a uniform share) with positive radiance, and a few
    records the trees must skip: zero, negative and non-finite radiance."""
    k = rng.integers(0, len(centres) + 1, n)
    d = _unit(rng.normal(size=(n, 3)))
    near = k < len(centres)
    d[near] = _unit(centres[k[near]] + spread * rng.normal(size=(int(near.sum()), 3)))
    r = rng.gamma(2.0, 1.0, n).astype(np.float32)
    if n == 0:
        return d.astype(np.float32), r
    bad = rng.choice(n, max(1, n // 50), replace=False)
    r[bad[0::3]] = 0.0
    r[bad[1::3]] = -1.0
    r[bad[2::3]] = np.nan
    return d.astype(np.float32), r


def _mine(pe, d1, r1, d2, r2, q, u):
    lib = pe._capi.load()
    pdf = np.zeros(len(q), np.float32)
    smp = np.zeros((len(q), 4), np.float32)
    pe._capi.check(lib.pe_sdtree_probe(_fp(d1), _fp(r1), len(r1), _fp(d2), _fp(r2), len(r2), _fp(q), _fp(u), len(q),
                                       pdf.ctypes.data_as(C.POINTER(C.c_float)),
                                       smp.ctypes.data_as(C.POINTER(C.c_float))))
    return pdf, smp


@pytest.mark.parametrize("seed,n1,n2,spread", [(0, 300, 2000, 0.15), (1, 5000, 20000, 0.05), (2, 40, 0, 0.3),
                                                 (3, 0, 0, 0.1)])
def test_quadtree_matches_reference(pe, oracle, seed, n1, n2, spread):
    rng = np.random.default_rng(seed)
    centres = _unit(rng.normal(size=(3, 3)))
    centres[0] = (0.0, 1.0, 0.0)      # the pole of the cylindrical map
    d1, r1 = _splats(rng, n1, centres, spread)
    d2, r2 = _splats(rng, n2, centres, spread)
    q = _unit(rng.normal(size=(4000, 3))).astype(np.float32)
    q[:3] = centres
    u = rng.uniform(0.0, 1.0, (4000, 2)).astype(np.float32)
    u[0] = (0.0, 0.0)
    u[1] = (1.0, 1.0)
    pdf, smp = _mine(pe, d1, r1, d2, r2, q, u)
    ref_pdf, ref_smp = oracle.dtree_probe(d1, r1, d2, r2, q, u)
    assert np.array_equal(pdf.view(np.uint32), ref_pdf.view(np.uint32))
    assert np.array_equal(smp.view(np.uint32), ref_smp.view(np.uint32))


def test_quadtree_is_a_density(pe):
    """Sampling and pdf agree, and the pdf integrates to one over the sphere."""
    rng = np.random.default_rng(5)
    centres = _unit(rng.normal(size=(2, 3)))
    d1, r1 = _splats(rng, 3000, centres, 0.1)
    d2, r2 = _splats(rng, 30000, centres, 0.1)
    n = 200000
    q = _unit(rng.normal(size=(n, 3))).astype(np.float32)
    u = rng.uniform(0.0, 1.0, (n, 2)).astype(np.float32)
    pdf, smp = _mine(pe, d1, r1, d2, r2, q, u)
    assert abs(pdf.mean() * 4.0 * np.pi - 1.0) < 2e-2, pdf.mean() * 4.0 * np.pi
    pdf_at, _ = _mine(pe, d1, r1, d2, r2, smp[:, :3], u)
    ok = smp[:, 3] > 0
    np.testing.assert_allclose(pdf_at[ok], smp[ok, 3], rtol=1e-3)
    # a trained tree concentrates (after two passes its cells are still 1/16 of the map wide):
    # samples land near a centre well more often than uniform directions do
    near = np.max(smp[:, :3] @ centres.T, axis=1) > np.cos(0.4)
    near_uniform = np.max(q @ centres.T, axis=1) > np.cos(0.4)
    assert near.mean() > 1.5 * near_uniform.mean(), (near.mean(), near_uniform.mean())
