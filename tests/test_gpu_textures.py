"""Image maps of the Disney material (DisneyMaterial::resolve, disney.cpp:543-603) on the CUDA
path against the reference engine's CPU path, same scene and Owen-Sobol indices:

* base colour, roughness (green channel), metalness (blue channel) and a tangent-space normal
  map, looked up bilinearly with wrap (Image::sampleLevel, image.cpp:168-225);
* UV mapping with a texture scale on a quad with vertex uvs (uv interpolation,
  triangle.cpp:107), and box projection on a sphere without uvs (textureCoord,
  disney.cpp:517-526).

Tolerance: as the other equal-spp parity renders, relMSE ≤ 1e-4 with ≥ 99 % of the pixels
equal to 1e-4 relative, and no bias.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes():
    return importlib.import_module("photon_engine_b200.scenes")


def _grid_quad(origin, u, v, n):
    """A quad of n×n cells with vertex uvs in [0, 1]²."""
    o, u, v = (np.asarray(x, np.float32) for x in (origin, u, v))
    s = np.linspace(0.0, 1.0, n + 1, dtype=np.float32)
    a, b = np.meshgrid(s, s, indexing="xy")
    pos = o + a[..., None] * u + b[..., None] * v
    uv = np.stack([a, b], axis=-1)
    idx = []
    for j in range(n):
        for i in range(n):
            k = j * (n + 1) + i
            idx += [k, k + 1, k + n + 2, k, k + n + 2, k + n + 1]
    return pos.reshape(-1, 3), uv.reshape(-1, 2), np.array(idx, np.uint32)


def _maps(seed=3):
    rng = np.random.default_rng(seed)
    cells = rng.uniform(0.05, 0.95, (4, 4, 3)).astype(np.float32)
    albedo = np.kron(cells, np.ones((8, 8, 1), np.float32))                    # 32×32 checker
    rough = np.zeros((16, 16, 3), np.float32)
    rough[..., 1] = rng.uniform(0.1, 0.9, (16, 16))
    metal = np.zeros((8, 8, 3), np.float32)
    metal[..., 2] = (rng.uniform(size=(8, 8)) > 0.5).astype(np.float32)
    y, x = np.mgrid[0:32, 0:32].astype(np.float32) / 32.0
    nx, ny = 0.35 * np.sin(2 * np.pi * 3 * x), 0.35 * np.cos(2 * np.pi * 2 * y)
    n = np.stack([nx, ny, np.ones_like(nx)], axis=-1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    normal = (n * 0.5 + 0.5).astype(np.float32)
    return albedo, rough, metal, normal


def test_image_maps_match_reference(pe, device, oracle):
    S = scenes()
    scene, cam, st = S.cornell_box(64, 64, 8, 6, seed=0)
    st.seed = 7
    albedo, rough, metal, normal = _maps()
    # a UV-mapped quad on the back wall, tiled twice
    m = pe.DisneyMaterial((0.5, 0.5, 0.5), 0.0, 0.5, 0.5)
    m.set_albedo_image(albedo)
    m.set_roughness_image(rough)
    m.set_metalness_image(metal)
    m.set_normal_image(normal)
    m.set_texture_scale(2.0)
    pos, uv, idx = _grid_quad((0.6, 0.6, 5.2), (4.4, 0.0, 0.0), (0.0, 4.4, 0.0), 4)
    scene.add_shape(pe.TriangleMesh(pos, None, uv, idx, m))
    # a box-projected sphere sharing the albedo image
    b = pe.DisneyMaterial((0.5, 0.5, 0.5), 0.0, 0.3, 0.5)
    b.set_albedo_image(albedo)
    b.set_normal_image(normal)
    b.set_texture_mapping(True)
    b.set_texture_scale(0.7)
    p, n, i = S.uv_sphere((3.8, 1.2, 2.2), 1.1, 48, 24)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, b))
    assert len(scene.textures()) == 4
    scene.build_accelerator()
    device.set_scene(scene)
    spp = 8
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, spp)
    mean_ref, cnt_ref = oracle.RefScene(scene).render(cam, st, 0, spp)
    assert np.array_equal(film.count, cnt_ref)
    img = film.resolve()
    err = pe.rel_mse(img, mean_ref)
    same = float(np.mean(np.all(np.abs(img - mean_ref) <= 1e-4 * np.maximum(1.0, np.abs(mean_ref)), axis=-1)))
    bias = float(img.mean() / max(1e-12, mean_ref.mean()) - 1.0)
    assert err < 1e-4 and same > 0.99 and abs(bias) < 1e-3, (err, same, bias)
    # the maps show: the same scene with plain materials renders differently
    plain = pe.Film(st.width, st.height)
    for mat in (m, b):
        mat.images.clear()
    scene.build_accelerator()
    device.set_scene(scene)
    device.render(cam, st, pe.RenderTargets(beauty=plain), 0, spp)
    assert pe.rel_mse(plain.resolve(), img) > 1e-3


def test_texture_index_is_checked(pe):
    lib = pe._capi.load()
    s = lib.pe_scene_create()
    try:
        m = pe.DisneyMaterial((0.5, 0.5, 0.5), 0.0, 0.5).struct
        m.albedo_texture = 0  # no texture added yet
        assert lib.pe_scene_add_material(s, m) < 0
        img = np.ones((2, 2, 3), np.float32)
        assert lib.pe_scene_add_texture(s, pe._capi.fptr(img), 2, 2) == 0
        assert lib.pe_scene_add_material(s, m) >= 0
    finally:
        lib.pe_scene_destroy(s)


def test_mipmapped_maps_match_reference(pe, device, oracle):
    """Mipmapped images (Image::buildMipmaps) looked up at the level of the ray cone's footprint
    (sampleTex, disney.cpp:530-539; cones path_tracer.cpp:428-454, 853-857): a receding floor
    whose far texels shrink below a pixel, seen directly and in a mirror."""
    S = scenes()
    scene = pe.Scene()
    rng = np.random.default_rng(5)
    checker = np.kron(rng.uniform(0.05, 0.95, (16, 16, 3)).astype(np.float32), np.ones((4, 4, 1), np.float32))
    floor = pe.DisneyMaterial((0.5, 0.5, 0.5), 0.0, 0.6, 0.5)
    floor.set_albedo_image(checker, mipmaps=True)
    floor.set_texture_scale(6.0)
    pos, uv, idx = _grid_quad((-20.0, 0.0, -2.0), (40.0, 0.0, 0.0), (0.0, 0.0, 60.0), 8)
    scene.add_shape(pe.TriangleMesh(pos, None, uv, idx, floor))
    p, n, i = S.uv_sphere((1.5, 1.0, 4.0), 1.0, 48, 24)
    scene.add_shape(pe.TriangleMesh(p, n, None, i, pe.Mirror((0.9, 0.9, 0.9))))
    scene.add_light(pe.AreaLight((-2.0, 6.0, 2.0), (4.0, 0.0, 0.0), (0.0, 0.0, 4.0), (12.0, 12.0, 12.0)))
    sky = np.ones((16, 32, 3), np.float32) * 0.5
    scene.set_environment(pe.EnvironmentLight(sky, 0.0, 1.0))
    cam = pe.PerspectiveCamera((0.0, 1.5, -1.5), (0.0, 0.5, 10.0), (0.0, 1.0, 0.0), 50.0, 1.0)
    st = pe.RenderSettings(width=64, height=64, max_bounces=4, seed=7)
    scene.build_accelerator()
    device.set_scene(scene)
    spp = 8
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, spp)
    mean_ref, cnt_ref = oracle.RefScene(scene).render(cam, st, 0, spp)
    img = film.resolve()
    err = pe.rel_mse(img, mean_ref)
    same = float(np.mean(np.all(np.abs(img - mean_ref) <= 1e-4 * np.maximum(1.0, np.abs(mean_ref)), axis=-1)))
    bias = float(img.mean() / max(1e-12, mean_ref.mean()) - 1.0)
    assert err < 1e-4 and same > 0.99 and abs(bias) < 1e-3, (err, same, bias)
    # the mip levels matter: without them the far floor aliases to other colours
    floor.mipmapped.clear()
    scene.build_accelerator()
    device.set_scene(scene)
    plain = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=plain), 0, spp)
    assert pe.rel_mse(plain.resolve(), img) > 1e-4


def test_opacity_map_matches_reference(pe, device, oracle):
    """DisneyMaterial::setOpacityImage: coverage = opacity × the map's red channel for camera
    and bounce rays (passesCutout, path_tracer.cpp:161-167) and for shadow rays
    (shadowTransmittance, disney.cpp:511-513)."""
    S = scenes()
    scene, cam, st = S.cornell_box(64, 64, 8, 6, seed=0)
    st.seed = 7
    y, x = np.mgrid[0:32, 0:32].astype(np.float32) / 32.0
    stripes = np.zeros((32, 32, 3), np.float32)
    stripes[..., 0] = np.where(np.sin(2 * np.pi * 5 * (x + 0.3 * y)) > 0.0, 1.0, 0.15)
    leaf = pe.DisneyMaterial((0.2, 0.6, 0.2), 0.0, 0.5, 0.5)
    leaf.set_opacity_image(stripes)
    pos, uv, idx = _grid_quad((0.8, 0.4, 1.2), (3.6, 0.0, 0.4), (0.0, 3.8, 0.0), 2)
    scene.add_shape(pe.TriangleMesh(pos, None, uv, idx, leaf))
    scene.build_accelerator()
    device.set_scene(scene)
    spp = 8
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, spp)
    mean_ref, cnt_ref = oracle.RefScene(scene).render(cam, st, 0, spp)
    img = film.resolve()
    err = pe.rel_mse(img, mean_ref)
    same = float(np.mean(np.all(np.abs(img - mean_ref) <= 1e-4 * np.maximum(1.0, np.abs(mean_ref)), axis=-1)))
    bias = float(img.mean() / max(1e-12, mean_ref.mean()) - 1.0)
    assert err < 1e-4 and same > 0.99 and abs(bias) < 1e-3, (err, same, bias)
    # the map shows: an opaque pane renders differently
    leaf.images.clear()
    scene.build_accelerator()
    device.set_scene(scene)
    opaque = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=opaque), 0, spp)
    assert pe.rel_mse(opaque.resolve(), img) > 1e-3


def test_8bit_images_match_reference(pe, device, oracle):
    """8-bit images (Image::createCompact8): an sRGB-encoded base colour with mipmaps (levels
    quantised to 8 bits, image.cpp:102-155) and a linear 8-bit roughness map, against the
    reference's lookups of the same bytes."""
    S = scenes()
    scene, cam, st = S.cornell_box(64, 64, 8, 6, seed=0)
    st.seed = 7
    rng = np.random.default_rng(9)
    albedo = np.kron(rng.integers(0, 256, (8, 8, 3)), np.ones((4, 4, 1), np.int64)).astype(np.uint8)
    rough = np.zeros((16, 16, 3), np.uint8)
    rough[..., 1] = rng.integers(20, 230, (16, 16))
    m = pe.DisneyMaterial((0.5, 0.5, 0.5), 0.0, 0.5, 0.5)
    m.set_albedo_image(albedo, mipmaps=True)
    m.set_roughness_image(rough)
    m.set_texture_scale(3.0)
    pos, uv, idx = _grid_quad((0.3, 0.01, 0.3), (4.9, 0.0, 0.0), (0.0, 0.0, 4.9), 4)
    scene.add_shape(pe.TriangleMesh(pos, None, uv, idx, m))
    scene.build_accelerator()
    device.set_scene(scene)
    spp = 8
    film = pe.Film(st.width, st.height)
    device.render(cam, st, pe.RenderTargets(beauty=film), 0, spp)
    mean_ref, _ = oracle.RefScene(scene).render(cam, st, 0, spp)
    img = film.resolve()
    err = pe.rel_mse(img, mean_ref)
    same = float(np.mean(np.all(np.abs(img - mean_ref) <= 1e-4 * np.maximum(1.0, np.abs(mean_ref)), axis=-1)))
    bias = float(img.mean() / max(1e-12, mean_ref.mean()) - 1.0)
    assert err < 1e-4 and same > 0.99 and abs(bias) < 1e-3, (err, same, bias)
