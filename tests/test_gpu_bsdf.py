"""Per-material BSDF parity: Material::evalPdf and Material::sampleFull of the device against
the reference's own materials at the same synthetic shading points.

Tolerance: eval f and pdf at given directions, 1e-5 relative (plus 1e-6 absolute near zero).
Sampled direction, f and pdf: 1e-4 relative — the sampled direction carries the ≤ 2 ulp
difference of CUDA's and glibc's sinf/cosf, and a steep GGX lobe (f ~ 1e3) amplifies that
into the 1e-5 range.  The sample's lobe flags must be equal.  Both sides evaluate the same
formulas with FMA contraction off.
"""
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-5, 1e-6


def materials(pe):
    out = {}
    out["lambert"] = pe.Lambertian((0.6, 0.4, 0.2))
    out["disney_plastic"] = pe.DisneyMaterial((0.8, 0.2, 0.1), 0.0, 0.4, 0.5)
    m = pe.DisneyMaterial((0.9, 0.7, 0.3), 1.0, 0.25, 0.5)
    m.set_edge_tint((0.8, 0.5, 0.3))
    out["disney_metal_f82"] = m
    m = pe.DisneyMaterial((0.2, 0.3, 0.8), 0.0, 0.6, 0.5)
    m.set_clear_coat(0.8)
    m.set_clear_coat_roughness(0.1)
    m.set_coat_tint((0.9, 0.95, 1.0))
    out["disney_clearcoat"] = m
    m = pe.DisneyMaterial((0.5, 0.1, 0.4), 0.0, 0.7, 0.3)
    m.set_sheen(0.9)
    m.set_sheen_roughness(0.4)
    m.set_diffuse_roughness(0.6)
    out["disney_sheen_eon"] = m
    m = pe.DisneyMaterial((0.7, 0.7, 0.7), 0.5, 0.3, 0.5)
    m.set_anisotropy(0.7)
    out["disney_aniso"] = m
    m = pe.DisneyMaterial((0.95, 0.95, 0.95), 0.0, 0.15, 0.5)
    m.set_specular_transmission(1.0)
    m.set_ior(1.45)
    out["disney_spec_trans"] = m
    m = pe.DisneyMaterial((0.3, 0.8, 0.3), 0.0, 0.5, 0.5)
    m.set_diffuse_transmission(0.6)
    out["disney_diff_trans"] = m
    m = pe.DisneyMaterial((0.6, 0.6, 0.6), 1.0, 0.2, 0.5)
    m.set_thin_film(420.0, 1.35)
    out["disney_thin_film"] = m
    m = pe.DisneyMaterial((0.1, 0.1, 0.4), 0.0, 0.5, 0.5)
    m.set_flakes(0.7, 0.05, 0.3, (0.9, 0.8, 0.6))
    out["disney_flakes"] = m
    m = pe.DisneyMaterial((0.9, 0.6, 0.5), 0.0, 0.5, 0.5)
    m.set_subsurface(0.8)
    out["disney_sss"] = m
    out["glass_smooth"] = pe.Dielectric(1.5, (1.0, 1.0, 1.0), 0.0)
    out["glass_rough"] = pe.Dielectric(1.5, (0.9, 0.95, 1.0), 0.3)
    g = pe.Dielectric(1.5, (1.0, 1.0, 1.0), 0.0)
    g.set_thin_walled(True)
    out["glass_thin"] = g
    g = pe.Dielectric(1.5, (1.0, 1.0, 1.0), 0.2)
    g.set_abbe(35.0)
    out["glass_dispersive"] = g
    out["mirror"] = pe.Mirror((0.9, 0.9, 0.85))
    return out


@pytest.fixture(scope="module")
def bsdf_scene(pe, device, oracle):
    mats = materials(pe)
    scene = pe.Scene()
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    for i, m in enumerate(mats.values()):
        scene.add_shape(pe.TriangleMesh(tri + np.float32(2 * i), None, None, np.array([[0, 1, 2]], np.uint32), m))
    scene.build_accelerator()
    device.set_scene(scene)
    ref = oracle.RefScene(scene)
    return mats, scene, ref


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def queries(pe, n, seed, back_face=False):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nrm = unit(rng.normal(size=3))
        t = unit(np.cross(nrm, unit(rng.normal(size=3))))
        wo = unit(rng.normal(size=3))
        if np.dot(wo, nrm) < 0:
            wo = -wo
        wi = unit(rng.normal(size=3))
        if i % 3 != 0 and np.dot(wi, nrm) < 0:
            wi = -wi  # two thirds reflection, one third transmission side
        q = pe._capi.pe_bsdf_query()
        q.wo = pe._capi.f3(wo)
        q.wi = pe._capi.f3(wi)
        q.normal = pe._capi.f3(nrm)
        q.ng = pe._capi.f3(-nrm if back_face else nrm)
        q.tangent = pe._capi.f3(t)
        q.point = pe._capi.f3(rng.uniform(-1, 1, 3))
        q.front_face = 0 if back_face else 1
        q.wavelength = float(rng.uniform(400, 700)) if i % 2 else 0.0
        q.uc = float(rng.uniform())
        q.u = (pe._capi.C.c_float * 2)(*rng.uniform(0, 1, 2))
        out.append(q)
    return out


RTOL_SAMPLE = 1e-4


def close(a, b, rtol=RTOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= ATOL + rtol * np.maximum(np.abs(a), np.abs(b)))


@pytest.mark.parametrize("name", [
    "lambert", "disney_plastic", "disney_metal_f82", "disney_clearcoat", "disney_sheen_eon", "disney_aniso",
    "disney_spec_trans", "disney_diff_trans", "disney_thin_film", "disney_flakes", "disney_sss", "glass_smooth",
    "glass_rough", "glass_thin", "glass_dispersive", "mirror"])
@pytest.mark.parametrize("back_face", [False, True])
def test_bsdf_eval_pdf_and_sample_match_reference(pe, device, bsdf_scene, name, back_face):
    mats, scene, ref = bsdf_scene
    m = mats[name]
    index = scene._mat_index[id(m)]
    q = queries(pe, 400, zlib.crc32(name.encode()) % 1000 + back_face, back_face)
    mine = device.bsdf_probe(index, q)
    theirs = ref.bsdf_probe(m, q, pe._capi.pe_bsdf_result)
    bad = []
    for i, (a, b) in enumerate(zip(mine, theirs)):
        ok = close(a.f[:], b.f[:]) and close(a.pdf, b.pdf) and a.sampled == b.sampled
        if ok and b.sampled:
            ok = (a.delta == b.delta and a.pass_through == b.pass_through and a.subsurface == b.subsurface and
                  close(a.wi[:], b.wi[:], RTOL_SAMPLE) and close(a.sf[:], b.sf[:], RTOL_SAMPLE) and
                  close(a.spdf, b.spdf, RTOL_SAMPLE) and close(a.weight[:], b.weight[:], RTOL_SAMPLE))
        if not ok:
            bad.append((i, list(a.f), a.pdf, list(b.f), b.pdf, a.sampled, b.sampled, list(a.sf), a.spdf, list(b.sf), b.spdf))
    assert not bad, f"{len(bad)} mismatches, first: {bad[:2]}"
