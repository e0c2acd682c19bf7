"""The photon engine's project files (``.photon``) on the B200 device.

``load_project(path, width, height)`` reads a project (JSON, format "photon-project", version ≥ 2)
and builds the render scene, camera and settings the reference builds from it, following
``loadProjectJson`` (src/scene/project_io.cpp:647-685), ``buildRenderScene``
(src/scene/document.cpp:315-352) and the CLI's ``cameraFromJson`` / render settings
(src/main.cpp:88-110, 222-260):

* materials (project_io.cpp:149-190): "glass" → Dielectric(ior, tint, roughness), "lambert" →
  Lambertian(albedo, emission), "mirror" → Mirror(color), anything else → DisneyMaterial with its
  scalar keys, emission, mapping and texture scale; then the advanced keys of a material preset
  (material_library.cpp:151-262: round edges, opacity, IOR, coat, sheen colour, EON roughness,
  subsurface, edge tint, thin film, flakes; for glass thin walls, absorption, scattering, Abbe);
* nodes (project_io.cpp:268-412, scene_graph.cpp:166-225): groups, "mesh" nodes with inline
  geometry (p, n, uv, i), "sphere" nodes; row-major 4×4 "xf" transforms composed parent × local;
  invisible nodes and their subtrees skipped; each mesh node a MeshInstance of its local mesh
  under the composed Transform (matrix parent·local, inverse local⁻¹·parent⁻¹, each node's inverse
  Mat4f::inverse of its "xf"), spheres as Sphere(world centre, radius × largest axis scale); the
  node's "visibility" ray mask on both;
* the automatic ground quad under the scene (scene_graph.cpp:151-165, document.cpp:327-343);
* area lights (document.cpp:67-117), temperature-free colour × intensity;
* the environment (project_io.cpp:543-583, document.cpp:118-140, 216-231): a Radiance .hdr
  image, else the procedural studio gradient, rotation in degrees, intensity (an environment of
  intensity 0 is left out); background mode and colour;
* the orbit camera (main.cpp:88-110): eye = target + r·(sin θ cos φ, cos θ, sin θ sin φ),
  perspective, thin lens or orthographic; float sin / cos / tan are the C library's.

Not carried (a ProjectError names the first one met): external meshes ("bin" files) and imported
model sources, point / spot / directional lights, the physical sky, image maps, camera shift,
motion (transform keys).
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import pathlib

import numpy as np

from . import engine as E


class ProjectError(ValueError):
    """A project the B200 device cannot render as the reference would."""


_libm = ctypes.CDLL("libm.so.6")
for _fn in ("sinf", "cosf", "tanf"):
    getattr(_libm, _fn).restype = ctypes.c_float
    getattr(_libm, _fn).argtypes = [ctypes.c_float]

F = np.float32
DEG_TO_RAD = F(math.pi) / F(180.0)
K_GROUND_NODE_UID = (1 << 64) - 2  # kGroundNodeUid of the reference's scene graph


def _vec3(j, key, default):
    v = j.get(key)
    if not isinstance(v, list) or len(v) < 3:
        return tuple(F(x) for x in default)
    return tuple(F(x) for x in v[:3])


def _mat_mul(a, b):
    """Mat4f::operator* (mat.h:57-67): row-by-column sums in order, in float32."""
    out = np.zeros((4, 4), F)
    for r in range(4):
        for c in range(4):
            out[r, c] = ((a[r, 0] * b[0, c] + a[r, 1] * b[1, c]) + a[r, 2] * b[2, c]) + a[r, 3] * b[3, c]
    return out


def _transform(j):
    """readTransform (project_io.cpp:94-101): Transform(m) of the node's "xf" (its inverse by
    Mat4f::inverse), or the identity Transform without one."""
    x = j.get("xf")
    if not isinstance(x, list) or len(x) != 16:
        return np.eye(4, dtype=F), np.eye(4, dtype=F)
    m = np.array(x, F).reshape(4, 4)
    inv = np.empty((4, 4), F)
    E._lib().pe_mat4_inverse(E.capi.fptr(np.ascontiguousarray(m)), E.capi.fptr(inv))
    return m, inv


def _points(m, p):
    """Transform::transformPoint (transform.cpp:15-26) of an (n, 3) float32 array."""
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    r = [((m[i, 0] * x + m[i, 1] * y) + m[i, 2] * z) + m[i, 3] * F(1.0) for i in range(4)]
    w = r[3]
    out = np.stack(r[:3], -1).astype(F)
    div = (w != F(1.0)) & (w != F(0.0))
    if div.any():
        inv = (F(1.0) / w[div]).astype(F)
        out[div] = out[div] * inv[:, None]
    return out


def _vectors(m, v):
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    return np.stack([(m[i, 0] * x + m[i, 1] * y) + m[i, 2] * z for i in range(3)], -1).astype(F)


def _procedural_sky(zenith, horizon):
    """makeProceduralSky (document.cpp:118-140): 512×256 zenith → horizon → ground gradient and two
    bright rectangles."""
    W, H = 512, 256
    z, h = np.array(zenith, F), np.array(horizon, F)
    img = np.zeros((H, W, 3), F)
    for y in range(H):
        t = F(y) / F(H - 1)
        if t < F(0.5):
            k = t * F(2.0)
            c = z * (F(1.0) - k) + h * k
        else:
            k = (t - F(0.5)) * F(2.0)
            c = h * (F(1.0) - F(0.65) * k)
        img[y, :] = c
    img[H * 14 // 100:H * 34 // 100, W * 40 // 100:W * 56 // 100] = (26.0, 25.0, 23.0)
    img[H * 22 // 100:H * 40 // 100, W * 6 // 100:W * 14 // 100] = (9.0, 10.0, 12.0)
    return img


def read_hdr(path) -> np.ndarray:
    """A Radiance RGBE (.hdr) image as float32 (h, w, 3), top row first: flat or run-length
    encoded scanlines, each texel mantissa · 2^(exponent − 136) (0 for a zero exponent)."""
    data = pathlib.Path(path).read_bytes()
    pos = 0
    header_end = data.find(b"\n\n")
    if not data.startswith(b"#?") or header_end < 0:
        raise ProjectError(f"{path}: not a Radiance HDR file")
    if b"FORMAT=32-bit_rle_rgbe" not in data[:header_end]:
        raise ProjectError(f"{path}: only 32-bit RGBE HDR files are read")
    pos = header_end + 2
    eol = data.index(b"\n", pos)
    dims = data[pos:eol].split()
    pos = eol + 1
    if len(dims) != 4 or dims[0] != b"-Y" or dims[2] != b"+X":
        raise ProjectError(f"{path}: unsupported HDR orientation {data[pos:eol]!r}")
    h, w = int(dims[1]), int(dims[3])
    rgbe = np.zeros((h, w, 4), np.uint8)
    buf = memoryview(data)
    for y in range(h):
        if 8 <= w < 32768 and buf[pos] == 2 and buf[pos + 1] == 2 and not (buf[pos + 2] & 0x80):
            if (buf[pos + 2] << 8 | buf[pos + 3]) != w:
                raise ProjectError(f"{path}: scanline width mismatch")
            pos += 4
            for c in range(4):
                x = 0
                while x < w:
                    n = buf[pos]
                    pos += 1
                    if n > 128:
                        n -= 128
                        rgbe[y, x:x + n, c] = buf[pos]
                        pos += 1
                    else:
                        rgbe[y, x:x + n, c] = np.frombuffer(buf[pos:pos + n], np.uint8)
                        pos += n
                    x += n
        else:
            rgbe[y] = np.frombuffer(buf[pos:pos + 4 * w], np.uint8).reshape(w, 4)
            pos += 4 * w
    e = rgbe[..., 3].astype(np.int32)
    scale = np.where(e > 0, np.ldexp(F(1.0), e - 136), F(0.0)).astype(F)
    return (rgbe[..., :3].astype(F) * scale[..., None]).astype(F)


def _material(j):
    """materialFromJson (project_io.cpp:149-190) + MaterialLibrary::applyAdvanced (material_library.cpp:151-177)."""
    t = j.get("type", "disney")
    adv = _advanced(j)
    if t == "glass":
        m = E.Dielectric(float(j.get("ior", 1.5)), _vec3(j, "tint", (1.0, 1.0, 1.0)), float(j.get("roughness", 0.0)))
        m.set_thin_walled(adv["thinWalled"])
        m.set_thin_film(adv["thinFilmThickness"] if adv["thinWalled"] else 0.0)
        if tuple(adv["absorbColor"]) != (1.0, 1.0, 1.0):
            m.set_absorption(adv["absorbColor"], adv["absorbDistance"])
        if adv["scatterDensity"] > 0.0:
            m.set_scattering(adv["scatterDensity"], adv["scatterColor"], adv["scatterAnisotropy"])
        m.set_abbe(max(adv["abbe"], 10.0) if adv["abbe"] > 0.0 else 0.0)
        m.set_round_edge_radius(adv["roundEdges"])
        return m
    if t == "lambert":
        m = E.Lambertian(_vec3(j, "albedo", (0.8, 0.8, 0.8)), _vec3(j, "emission", (0.0, 0.0, 0.0)))
        m.set_round_edge_radius(adv["roundEdges"])
        return m
    if t == "mirror":
        m = E.Mirror(_vec3(j, "color", (0.95, 0.95, 0.95)))
        m.set_round_edge_radius(adv["roundEdges"])
        return m
    if j.get("maps"):
        raise ProjectError("image maps of project materials are not read (the image decoders are not part of this build)")
    m = E.DisneyMaterial(_vec3(j, "baseColor", (0.8, 0.8, 0.8)), float(j.get("metallic", 0.0)),
                         float(j.get("roughness", 0.5)), float(j.get("specular", 0.5)))
    m.set_clear_coat(float(j.get("clearCoat", 0.0)))
    m.set_clear_coat_roughness(float(j.get("clearCoatRoughness", 0.03)))
    m.set_anisotropy(float(j.get("anisotropy", 0.0)))
    m.set_sheen(float(j.get("sheen", 0.0)))
    m.set_diffuse_transmission(float(j.get("diffuseTransmission", 0.0)))
    m.set_emission(_vec3(j, "emission", (0.0, 0.0, 0.0)))
    m.set_texture_mapping(j.get("mapping", "uv") == "box")
    m.set_texture_scale(float(j.get("texScale", 1.0)))
    m.set_opacity(adv["opacity"])
    m.set_ior(adv["ior"])
    m.set_specular_transmission(adv["specularTransmission"])
    m.set_coat_ior(adv["coatIor"])
    m.set_coat_tint(adv["coatTint"])
    if adv["hasCustomSheenColor"]:
        m.set_sheen_color(adv["sheenColor"])
    m.set_diffuse_roughness(adv["diffuseRoughness"])
    m.set_sheen_roughness(adv["sheenRoughness"])
    m.set_subsurface(adv["subsurface"])
    m.set_subsurface_radius(adv["subsurfaceRadius"])
    m.set_subsurface_scale(adv["subsurfaceScale"])
    m.set_subsurface_anisotropy(adv["subsurfaceAnisotropy"])
    m.set_edge_tint(adv["edgeTint"])
    m.set_thin_film(adv["thinFilmThickness"], adv["thinFilmIor"])
    if adv["flakeDensity"] > 0.0:
        m.set_flakes(adv["flakeDensity"], adv["flakeSize"], adv["flakeRoughness"], adv["flakeColor"])
    m.set_round_edge_radius(adv["roundEdges"])
    return m


def _advanced(j):
    """presetAdvancedFromJson (material_library.cpp:219-262) over MaterialPreset's defaults."""
    p = {"opacity": 1.0, "ior": 1.5, "specularTransmission": 0.0, "coatIor": 1.5, "coatTint": (1.0, 1.0, 1.0),
         "sheenColor": (1.0, 1.0, 1.0), "hasCustomSheenColor": False, "absorbColor": (1.0, 1.0, 1.0),
         "absorbDistance": 1.0, "scatterDensity": 0.0, "scatterColor": (1.0, 1.0, 1.0), "scatterAnisotropy": 0.0,
         "abbe": 0.0, "subsurface": 0.0, "subsurfaceRadius": (1.0, 0.2, 0.1), "subsurfaceScale": 0.05,
         "subsurfaceAnisotropy": 0.0, "edgeTint": (1.0, 1.0, 1.0), "diffuseRoughness": 0.0, "sheenRoughness": 0.3,
         "roundEdges": 0.0, "thinWalled": False, "thinFilmThickness": 0.0, "thinFilmIor": 1.4, "flakeDensity": 0.0,
         "flakeSize": 0.004, "flakeRoughness": 0.3, "flakeColor": (0.9, 0.9, 0.9)}
    for k in ("opacity", "ior", "specularTransmission", "coatIor", "abbe", "diffuseRoughness", "sheenRoughness",
              "roundEdges"):
        if k in j:
            p[k] = float(j[k])
    for k in ("coatTint", "edgeTint"):
        p[k] = _vec3(j, k, p[k])
    if "sheenColor" in j:
        p["sheenColor"] = _vec3(j, "sheenColor", p["sheenColor"])
        p["hasCustomSheenColor"] = True
    if isinstance(j.get("absorption"), dict):
        a = j["absorption"]
        p["absorbColor"] = _vec3(a, "color", p["absorbColor"])
        p["absorbDistance"] = float(a.get("distance", p["absorbDistance"]))
    if isinstance(j.get("scattering"), dict):
        s = j["scattering"]
        p["scatterDensity"] = float(s.get("density", p["scatterDensity"]))
        p["scatterColor"] = _vec3(s, "color", p["scatterColor"])
        p["scatterAnisotropy"] = float(s.get("anisotropy", p["scatterAnisotropy"]))
    if isinstance(j.get("subsurface"), dict):
        s = j["subsurface"]
        p["subsurface"] = float(s.get("weight", p["subsurface"]))
        p["subsurfaceRadius"] = _vec3(s, "radius", p["subsurfaceRadius"])
        p["subsurfaceScale"] = float(s.get("scale", p["subsurfaceScale"]))
        p["subsurfaceAnisotropy"] = float(s.get("anisotropy", p["subsurfaceAnisotropy"]))
    if "thinWalled" in j:
        p["thinWalled"] = bool(j["thinWalled"])
    if isinstance(j.get("thinFilm"), dict):
        t = j["thinFilm"]
        p["thinFilmThickness"] = float(t.get("thickness", p["thinFilmThickness"]))
        p["thinFilmIor"] = float(t.get("ior", p["thinFilmIor"]))
    if isinstance(j.get("flakes"), dict):
        f = j["flakes"]
        p["flakeDensity"] = float(f.get("density", p["flakeDensity"]))
        p["flakeSize"] = float(f.get("size", p["flakeSize"]))
        p["flakeRoughness"] = float(f.get("roughness", p["flakeRoughness"]))
        p["flakeColor"] = _vec3(f, "color", p["flakeColor"])
    return p


class _Graph:
    """The scene graph of a project: compiled into a Scene in depth-first node order."""

    def __init__(self, nodes, materials):
        self.nodes = nodes
        self.materials = materials
        self.lo = np.full(3, np.inf, F)
        self.hi = np.full(3, -np.inf, F)
        self.count = 0

    def _merge(self, p):
        self.lo = np.minimum(self.lo, p.min(0)).astype(F)
        self.hi = np.maximum(self.hi, p.max(0)).astype(F)

    def compile(self, scene, j, parent, parent_inv):
        if j.get("source") is not None:
            raise ProjectError("imported model sources (\"source\" nodes) are not read")
        if "transformKeys" in j:
            raise ProjectError("animated node transforms are not carried")
        if not j.get("visible", True):
            return
        local, local_inv = _transform(j)
        world = _mat_mul(parent, local)              # Transform::operator* (transform.cpp:117-122)
        world_inv = _mat_mul(local_inv, parent_inv)
        vis = int(j.get("visibility", E.VIS_ALL)) & E.VIS_ALL
        mi = j.get("material", -1)
        mat = self.materials[mi] if isinstance(mi, int) and 0 <= mi < len(self.materials) else None
        kind = j.get("type", "group")
        name = j.get("name", "")
        if kind == "mesh":
            g = j.get("geometry", {})
            if "bin" in g:
                raise ProjectError("external mesh files (\"bin\" geometry) are not read")
            p = np.array(g.get("p", []), F).reshape(-1, 3)
            n = np.array(g.get("n", []), F).reshape(-1, 3)
            uv = np.array(g.get("uv", []), F).reshape(-1, 2)
            idx = np.array(g.get("i", []), np.int64)
            if p.size == 0 or idx.size % 3 != 0 or (idx.size and idx.max() >= p.shape[0]):
                return  # meshFromJson rejects the node
            self._merge(_points(world, p))
            if mat is not None:
                mesh = E.TriangleMesh(p, n if n.shape[0] == p.shape[0] else None,
                                      uv if uv.shape[0] == p.shape[0] else None, idx.astype(np.uint32).reshape(-1, 3), mat)
                inst = E.MeshInstance(mesh, world, mat, world_inv)
                inst.set_visibility_mask(vis)
                scene.add_shape(inst)
                self._name(scene, name, mat)
        elif kind == "sphere":
            r = float(j.get("radius", 1.0))
            c = _points(world, np.zeros((1, 3), F))[0]
            if r > 0:
                self._merge(np.stack([c - F(r), c + F(r)]))  # nodeWorldBounds: the unscaled radius
            if mat is not None and r > 0:
                axes = _vectors(world, np.eye(3, dtype=F))
                s = max(float(np.sqrt(np.float32(np.dot(a, a)))) for a in axes)
                sphere = E.Sphere(tuple(float(x) for x in c), float(F(r) * F(s)), mat)
                sphere.set_visibility_mask(vis)
                scene.add_shape(sphere)
                self._name(scene, name, mat)
        for child in j.get("children", []):
            self.compile(scene, child, world, world_inv)

    def _name(self, scene, name, mat):
        shape = scene.shape_count() - 1
        scene.set_shape_name(shape, name)
        if id(mat) not in scene.material_names:
            scene.set_material_name(mat, name + "_Mat")


def load_project(path, width: int = 512, height: int = 512, spp: int = 64):
    """(Scene, camera, RenderSettings) of a .photon project, as the reference's loader and
    buildRenderScene make them; ProjectError for what the device does not carry."""
    path = pathlib.Path(path)
    root = json.loads(path.read_text(encoding="utf-8"))
    if not isinstance(root, dict) or int(root.get("version", 0)) < 2:
        raise ProjectError(f"{path}: not a photon project of version 2 or later")
    base = path.resolve().parent
    materials = [_material(m) for m in root.get("materials", [])]
    scene = E.Scene()
    graph = _Graph(root.get("nodes", []), materials)
    for n in graph.nodes:
        graph.compile(scene, n, np.eye(4, dtype=F), np.eye(4, dtype=F))
    env = root.get("environment", {})
    if env.get("kind", "image") == "sky":
        raise ProjectError("the physical sky environment is not carried")
    ground = env.get("ground", {}) if isinstance(env.get("ground"), dict) else {}
    if ground.get("enabled", True) and np.isfinite(graph.lo).all() and (graph.lo[0] <= graph.hi[0]):
        lo, hi = graph.lo, graph.hi
        d = hi - lo
        span = max(float(d[0]), float(d[2]), float(d[1]), 1e-3)
        span = F(span)
        pad = span * F(100.0)
        cx = (lo[0] + hi[0]) * F(0.5)
        cz = (lo[2] + hi[2]) * F(0.5)
        corner = np.array([cx - pad, lo[1] - span * F(0.0005), cz - pad], F)
        eu = np.array([pad * F(2.0), 0.0, 0.0], F)
        ev = np.array([0.0, 0.0, pad * F(2.0)], F)
        p0, p1 = corner, corner + eu
        p2, p3 = p1 + ev, corner + ev
        gm = E.DisneyMaterial(_vec3(ground, "color", (0.42, 0.42, 0.42)), 0.0, float(ground.get("roughness", 0.55)), 0.5)
        scene.add_shape(E.TriangleMesh(np.stack([p0, p1, p2, p3]).astype(F), None, None,
                                       np.array([[0, 2, 1], [0, 3, 2]], np.uint32), gm))
        shape = scene.shape_count() - 1
        scene.tag_shape(shape, K_GROUND_NODE_UID)
        scene.set_shape_name(shape, "Zemin")
        if ground.get("shadowCatcher", False):
            scene.set_shadow_catcher(shape)
    for lj in root.get("lights", []):
        _light(scene, lj)
    intensity = float(env.get("intensity", 1.0))
    if intensity > 0.0:
        hdr = env.get("hdr", "")
        img = None
        if hdr:
            hp = pathlib.Path(hdr)
            hp = hp if hp.is_absolute() else base / hp
            if hp.exists():
                img = read_hdr(os.path.normpath(hp))
        if img is None:
            img = _procedural_sky(_vec3(env, "zenith", (0.75, 0.8, 0.95)), _vec3(env, "horizon", (0.55, 0.55, 0.58)))
        scene.set_environment(E.EnvironmentLight(img, float(F(float(env.get("rotation", 0.0))) * DEG_TO_RAD), intensity))
    bg = env.get("background", {}) if isinstance(env.get("background"), dict) else {}
    mode = bg.get("mode", "environment")
    scene.set_background(E.Background({"color": E.BackgroundMode.Color, "transparent": E.BackgroundMode.Transparent}
                                      .get(mode, E.BackgroundMode.Environment),
                                      _vec3(bg, "color", (0.18, 0.18, 0.18))))
    camera = _camera(root.get("camera", {}), width / height)
    render = root.get("render", {}) if isinstance(root.get("render"), dict) else {}
    fname = render.get("pixelFilter", "box")
    ftype = {"box": E.PixelFilterType.Box, "triangle": E.PixelFilterType.Triangle, "tent": E.PixelFilterType.Triangle,
             "gaussian": E.PixelFilterType.Gaussian, "gauss": E.PixelFilterType.Gaussian,
             "blackman-harris": E.PixelFilterType.BlackmanHarris, "bh": E.PixelFilterType.BlackmanHarris}.get(fname)
    if ftype is None:
        raise ProjectError(f"unknown pixel filter {fname!r}")
    settings = E.RenderSettings(width=width, height=height, samples_per_pixel=spp,
                                max_bounces=int(render.get("maxBounces", 8)), filter_type=ftype,
                                filter_width=float(render.get("filterWidth", 1.0 if ftype == E.PixelFilterType.Box else 1.5)),
                                clamp_indirect=float(render.get("clampIndirect", 0.0)),
                                path_guiding=bool(render.get("pathGuiding", False)))
    return scene, camera, settings


def _light(scene, j):
    """lightFromJson (project_io.cpp:474-518) + buildLights (document.cpp:67-117) for area lights."""
    t = j.get("type", "area")
    if not j.get("enabled", True) or float(j.get("intensity", 10.0)) <= 0.0:
        return
    if t != "area":
        raise ProjectError(f"{t} lights are not carried (area lights only)")
    if float(j.get("temperature", 0.0)) > 0.0:
        raise ProjectError("colour temperatures of lights are not carried")
    if j.get("lightLink"):
        raise ProjectError("light links of project lights are not carried")
    color = np.array(_vec3(j, "color", (1.0, 1.0, 1.0)), F)
    L = color * F(float(j.get("intensity", 10.0)))
    pos = np.array(_vec3(j, "position", (0.0, 3.0, 0.0)), F)
    tgt = np.array(_vec3(j, "target", (0.0, 0.0, 0.0)), F)
    n = tgt - pos
    if float(np.dot(n, n)) < 1e-12:
        n = np.array([0.0, -1.0, 0.0], F)
    n = (n / F(np.sqrt(F(np.dot(n, n))))).astype(F)
    up = np.array([1.0, 0.0, 0.0], F) if abs(n[1]) > 0.95 else np.array([0.0, 1.0, 0.0], F)
    u = np.cross(up, n).astype(F)
    u = (u / F(np.sqrt(F(np.dot(u, u))))).astype(F)
    v = np.cross(n, u).astype(F)
    v = (v / F(np.sqrt(F(np.dot(v, v))))).astype(F)
    u = u * F(max(1e-4, float(j.get("width", 1.0))))
    v = v * F(max(1e-4, float(j.get("height", 1.0))))
    corner = pos - u * F(0.5) - v * F(0.5)
    a = E.AreaLight(tuple(map(float, corner)), tuple(map(float, u)), tuple(map(float, v)), tuple(map(float, L)))
    a.set_visible_to_camera(bool(j.get("visibleToCamera", True)))
    if j.get("lightGroup"):
        a.set_light_group(j["lightGroup"])
    scene.add_light(a)


def _camera(c, aspect):
    """cameraFromJson (main.cpp:88-110)."""
    t = c.get("target")
    target = np.array(t, F) if isinstance(t, list) and len(t) == 3 else np.array([0.0, 0.5, 0.0], F)
    r, th, ph = F(c.get("radius", 5.0)), F(c.get("theta", 1.15)), F(c.get("phi", 0.45))
    fov = float(F(c.get("fov", 35.0)))
    if float(c.get("shiftX", 0.0)) != 0.0 or float(c.get("shiftY", 0.0)) != 0.0:
        raise ProjectError("camera shift is not carried")
    st, ct = F(_libm.sinf(th)), F(_libm.cosf(th))
    sp, cp = F(_libm.sinf(ph)), F(_libm.cosf(ph))
    d = np.array([st * cp, ct, st * sp], F)
    eye = (target + d * r).astype(F)
    eye_t = tuple(float(x) for x in eye)
    tgt_t = tuple(float(x) for x in target)
    if c.get("orthographic", False):
        h = F(2.0) * F(_libm.tanf(F(F(fov) * DEG_TO_RAD * F(0.5)))) * r
        return E.OrthographicCamera(eye_t, tgt_t, (0.0, 1.0, 0.0), float(h), aspect)
    aperture = float(c.get("aperture", 0.0))
    if aperture > 0.0:
        focus = float(c.get("focusDistance", r)) if c.get("focusExplicit", False) else float(r)
        return E.ThinLensCamera(eye_t, tgt_t, (0.0, 1.0, 0.0), fov, aspect, aperture, focus,
                                int(c.get("apertureBlades", 0)), float(c.get("bladeRotation", 0.0)))
    return E.PerspectiveCamera(eye_t, tgt_t, (0.0, 1.0, 0.0), fov, aspect)
