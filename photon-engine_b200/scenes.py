"""Seeded procedural scenes for the workloads the tracer is measured on.

No public dataset is involved: the reference measures on its own scenes, and these synthetic
scenes stand in for them with the stated sizes and value distributions.

* ``cornell_box``      36 triangles: five Lambert walls, an emissive ceiling quad (17, 12, 4),
                       two rotated boxes; 256², 64 spp, depth 8 in the plain CPU-runnable case.
* ``torus_knot_scene`` (2,3) torus knot of ~1M triangles with eight Disney materials assigned
                       to random face clusters (metallic ∈ {0,1}, roughness ~ U(0.05, 0.9),
                       clearcoat ~ U(0,1), base ~ U(0,1)³), a ground plane, a 2048×1024 float32
                       sky-gradient environment whose sun lobe holds 60 % of the power, and one
                       rectangular softbox; 1920×1080, 256 spp, depth 12 at product scale.
* ``media_scene``      many lights and media, in millimetres: a seeded spiral LED strip of 1000
                       quads (2000 emissive triangles, light-BVH NEE), a dispersive glass sphere
                       (IOR 1.5, Abbe 35), an absorbing liquid cylinder (σa ~ U(0.1, 2)/mm per
                       channel), a Henyey–Greenstein scattering sphere (g = 0.6) and a random-walk
                       subsurface slab (mean free path 1–5 mm); ~200k triangles, 1280×720,
                       512 spp, depth 24 at full size.
* ``room_scene``       indirect-lit interior: a closed 10×8×3 m room whose only opening is a
                       1×1 m window in the sun-facing wall, lit by the knot scene's sky; three
                       Disney torus knots, a sphere and tables on the floor (~0.5M triangles);
                       1920×1080 at full size.  The learned proposal's workload.
* ``instanced_grid_scene`` a 5×4 grid of 20 seeded MeshInstances of one 262k-triangle torus
                       knot (5.2M triangles seen, one BLAS of 262k stored), eight Disney
                       materials, the sky of the knot scene.
"""
from __future__ import annotations

import math

import numpy as np

from . import _capi as capi
from . import scenegen
from .engine import (AreaLight, Dielectric, DisneyMaterial, EnvironmentLight, Lambertian, Material, MeshInstance, Mirror,
                     PerspectiveCamera, PixelFilterType, RenderSettings, Scene, TriangleMesh)


CAMERAS = scenegen.CAMERAS


def camera_for(name: str, width: int, height: int) -> PerspectiveCamera:
    pos, target, up, fov = CAMERAS[name]
    return PerspectiveCamera(pos, target, up, fov, width / height)


def _quad(p0, p1, p2, p3):
    pos = np.array([p0, p1, p2, p3], np.float32)
    idx = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    return pos, idx


def _box(center, size, angle_deg):
    """Axis box rotated about +y, 4 vertices per face (flat vertex normals), 12 triangles."""
    cx, cy, cz = center
    sx, sy, sz = (s * 0.5 for s in size)
    a = math.radians(angle_deg)
    c, s = math.cos(a), math.sin(a)

    def P(x, y, z):
        return (cx + c * x + s * z, cy + y, cz - s * x + c * z)

    faces = [
        [P(-sx, -sy, -sz), P(-sx, sy, -sz), P(sx, sy, -sz), P(sx, -sy, -sz)],   # -z
        [P(sx, -sy, sz), P(sx, sy, sz), P(-sx, sy, sz), P(-sx, -sy, sz)],       # +z
        [P(-sx, -sy, sz), P(-sx, sy, sz), P(-sx, sy, -sz), P(-sx, -sy, -sz)],   # -x
        [P(sx, -sy, -sz), P(sx, sy, -sz), P(sx, sy, sz), P(sx, -sy, sz)],       # +x
        [P(-sx, sy, -sz), P(-sx, sy, sz), P(sx, sy, sz), P(sx, sy, -sz)],       # +y
        [P(-sx, -sy, sz), P(-sx, -sy, -sz), P(sx, -sy, -sz), P(sx, -sy, sz)],   # -y
    ]
    pos = np.array([v for f in faces for v in f], np.float32)
    idx = np.array([[4 * k, 4 * k + 1, 4 * k + 2] for k in range(6)] + [[4 * k, 4 * k + 2, 4 * k + 3] for k in range(6)],
                   np.uint32)
    return pos, idx


def cornell_box(width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8, seed: int = 0):
    """The plain CPU-runnable workload: 36 triangles, Lambert only, emissive ceiling quad."""
    W, H, D = 5.56, 5.488, 5.592
    white = Lambertian((0.73, 0.73, 0.73))
    red = Lambertian((0.65, 0.05, 0.05))
    green = Lambertian((0.12, 0.45, 0.15))
    light = Lambertian((0.0, 0.0, 0.0), emission=(17.0, 12.0, 4.0))
    scene = Scene()
    walls = [
        (_quad((0, 0, 0), (0, 0, D), (W, 0, D), (W, 0, 0)), white),      # floor
        (_quad((0, H, 0), (W, H, 0), (W, H, D), (0, H, D)), white),      # ceiling
        (_quad((0, 0, D), (0, H, D), (W, H, D), (W, 0, D)), white),      # back
        (_quad((W, 0, 0), (W, 0, D), (W, H, D), (W, H, 0)), green),      # right
        (_quad((0, 0, 0), (0, H, 0), (0, H, D), (0, 0, D)), red),        # left
    ]
    for (pos, idx), mat in walls:
        scene.add_shape(TriangleMesh(pos, None, None, idx, mat))
    lp, li = _quad((2.13, H - 0.01, 2.27), (3.43, H - 0.01, 2.27), (3.43, H - 0.01, 3.32), (2.13, H - 0.01, 3.32))
    scene.add_shape(TriangleMesh(lp, None, None, li, light))
    for center, size, ang in (((1.85, 0.825, 1.69), (1.65, 1.65, 1.65), -18.0),
                              ((3.68, 1.65, 3.51), (1.65, 3.3, 1.65), 15.0)):
        pos, idx = _box(center, size, ang)
        scene.add_shape(TriangleMesh(pos, None, None, idx, white))
    camera = camera_for("cornell", width, height)
    settings = RenderSettings(width=width, height=height, samples_per_pixel=spp, max_bounces=max_depth,
                              filter_type=PixelFilterType.Box, filter_width=1.0, seed=seed)
    return scene, camera, settings


torus_knot_mesh = scenegen.knot_mesh
sky_environment = scenegen.sky_image

_MATERIAL_CLASSES = {scenegen.MAT_LAMBERT: Lambertian, scenegen.MAT_DISNEY: DisneyMaterial,
                     scenegen.MAT_DIELECTRIC: Dielectric, scenegen.MAT_MIRROR: Mirror}


def material_from_description(d: dict) -> Material:
    """A product material from a description dict: pe_material_defaults of its type, then each
    named pe_material field."""
    cls = _MATERIAL_CLASSES[int(d["type"])]
    m = cls.__new__(cls)
    Material.__init__(m)
    for key, value in d.items():
        if key == "type":
            continue
        setattr(m.struct, key, capi.f3(value) if isinstance(value, (tuple, list, np.ndarray)) else value)
    return m


def from_description(desc: dict):
    """(Scene, PerspectiveCamera, RenderSettings) of a scenegen description."""
    mats = [material_from_description(m) for m in desc["materials"]]
    scene = Scene()
    for kind, o in desc["ops"]:
        if kind == "mesh":
            scene.add_shape(TriangleMesh(o["positions"], o.get("normals"), o.get("uvs"), o["indices"],
                                         mats[o["material"]]))
        else:
            scene.add_light(AreaLight(o["position"], o["u"], o["v"], o["radiance"]))
    env = desc.get("environment")
    if env is not None:
        scene.set_environment(EnvironmentLight(env["image"], env["rotation"], env["intensity"]))
    c = desc["camera"]
    camera = PerspectiveCamera(c["position"], c["target"], c["up"], c["vfov"], c["aspect"])
    st = dict(desc["settings"])
    st["filter_type"] = PixelFilterType(st["filter_type"])
    return scene, camera, RenderSettings(**st)


def torus_knot_scene(width: int = 1920, height: int = 1080, spp: int = 256, max_depth: int = 12, nu: int = 4096,
                     nv: int = 128, env_size=(2048, 1024), seed: int = 7, clusters: int = 64):
    """Product-scale workload: ~1M-triangle torus knot, eight Disney materials, HDR sky, softbox
    (``scenegen.torus_knot``)."""
    return from_description(scenegen.torus_knot(width, height, spp, max_depth, nu, nv, env_size, seed, clusters))


def uv_sphere(center, radius: float, nu: int, nv: int):
    """Latitude-longitude sphere with smooth vertex normals, wound outward: nu·(nv−1)·2 triangles."""
    cx, cy, cz = center
    th = np.linspace(0.0, math.pi, nv + 1)
    ph = np.linspace(0.0, 2.0 * math.pi, nu + 1)[:-1]
    st, ct = np.sin(th)[:, None], np.cos(th)[:, None]
    n = np.stack([st * np.cos(ph)[None, :], np.broadcast_to(ct, (nv + 1, nu)), st * np.sin(ph)[None, :]], -1)
    n = n.reshape(-1, 3)
    pos = (n * radius + np.array([cx, cy, cz])).astype(np.float32)
    tris = []
    for i in range(nv):
        a = i * nu + np.arange(nu)
        b = i * nu + (np.arange(nu) + 1) % nu
        c = (i + 1) * nu + (np.arange(nu) + 1) % nu
        d = (i + 1) * nu + np.arange(nu)
        if i > 0:
            tris.append(np.stack([a, b, c], -1))
        if i < nv - 1:
            tris.append(np.stack([a, c, d], -1))
    return pos, n.astype(np.float32), np.concatenate(tris).astype(np.uint32)


def cylinder(center, radius: float, height: float, nseg: int, nrings: int):
    """Closed cylinder about +y (base at center.y): smooth side normals, flat caps, wound outward
    (the geometric normal decides which side of a volume boundary a path is on)."""
    cx, cy, cz = center
    ph = np.linspace(0.0, 2.0 * math.pi, nseg + 1)[:-1]
    ring = np.stack([np.cos(ph), np.zeros_like(ph), np.sin(ph)], -1)
    ys = np.linspace(0.0, height, nrings + 1)
    side = np.concatenate([ring * radius + np.array([cx, cy + y, cz]) for y in ys])
    side_n = np.tile(ring, (nrings + 1, 1))
    tris = []
    for i in range(nrings):
        a = i * nseg + np.arange(nseg)
        b = i * nseg + (np.arange(nseg) + 1) % nseg
        tris.append(np.stack([a, b + nseg, b], -1))
        tris.append(np.stack([a, a + nseg, b + nseg], -1))
    pos, nrm, idx = [side], [side_n], [np.concatenate(tris)]
    base = side.shape[0]
    for y, sgn in ((0.0, -1.0), (height, 1.0)):
        rim = ring * radius + np.array([cx, cy + y, cz])
        centre = np.array([[cx, cy + y, cz]])
        pos.append(np.concatenate([centre, rim]))
        nrm.append(np.tile([0.0, sgn, 0.0], (nseg + 1, 1)))
        k = np.arange(nseg)
        a, b = base + 1 + k, base + 1 + (k + 1) % nseg
        c0 = np.full(nseg, base)
        idx.append(np.stack([c0, b, a], -1) if sgn > 0 else np.stack([c0, a, b], -1))
        base += nseg + 1
    return (np.concatenate(pos).astype(np.float32), np.concatenate(nrm).astype(np.float32),
            np.concatenate(idx).astype(np.uint32))


def grid_box(center, size, n: int):
    """Axis-aligned box whose faces are n×n quad grids (flat normals): 12·n² triangles."""
    c = np.asarray(center, np.float64)
    h = np.asarray(size, np.float64) * 0.5
    t = np.linspace(-1.0, 1.0, n + 1)
    pos, nrm, idx = [], [], []
    base = 0
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            u_ax, v_ax = [a for a in range(3) if a != axis]
            if sgn < 0:
                u_ax, v_ax = v_ax, u_ax
            uu, vv = np.meshgrid(t, t, indexing="ij")
            p = np.zeros((n + 1, n + 1, 3))
            p[..., axis] = sgn
            p[..., u_ax] = uu
            p[..., v_ax] = vv
            p = p.reshape(-1, 3) * h + c
            nn = np.zeros((p.shape[0], 3))
            nn[:, axis] = sgn
            i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
            a = (i * (n + 1) + j).ravel() + base
            b = a + (n + 1)
            tri = np.concatenate([np.stack([a, b, b + 1], -1), np.stack([a, b + 1, a + 1], -1)])
            # outward winding: the geometric normal must agree with the face normal
            e = np.cross(p[tri[:, 1] - base] - p[tri[:, 0] - base], p[tri[:, 2] - base] - p[tri[:, 0] - base])
            if np.dot(e[0], nn[0]) < 0:
                tri = tri[:, [0, 2, 1]]
            pos.append(p)
            nrm.append(nn)
            idx.append(tri)
            base += p.shape[0]
    return (np.concatenate(pos).astype(np.float32), np.concatenate(nrm).astype(np.float32),
            np.concatenate(idx).astype(np.uint32))


def led_strip(n_quads: int, seed: int, height: float = 350.0, r0: float = 60.0, r1: float = 620.0,
              turns: float = 3.2, size: float = 9.0):
    """Spiral of downward-facing emissive quads (2 triangles each) above the floor."""
    rng = np.random.default_rng(seed)
    t = (np.arange(n_quads) + 0.5) / n_quads
    a = 2.0 * math.pi * turns * t + rng.uniform(-0.01, 0.01, n_quads)
    r = r0 + (r1 - r0) * t
    cx, cz = r * np.cos(a), r * np.sin(a)
    tx, tz = -np.sin(a), np.cos(a)          # along the strip
    h = size * 0.5
    rx, rz = np.cos(a), np.sin(a)           # across the strip (radial)
    pos = np.zeros((n_quads, 4, 3))
    for k, (su, sv) in enumerate(((-1, -1), (1, -1), (1, 1), (-1, 1))):
        pos[:, k, 0] = cx + su * h * tx + sv * h * rx
        pos[:, k, 2] = cz + su * h * tz + sv * h * rz
        pos[:, k, 1] = height
    # (0, 2, 1), (0, 3, 2): tangent × radial is +y, so this winding faces the floor
    idx = np.arange(n_quads)[:, None] * 4 + np.array([[0, 2, 1], [0, 3, 2]]).reshape(1, 2, 3).transpose(1, 0, 2)
    idx = np.concatenate([idx[0], idx[1]])
    return pos.reshape(-1, 3).astype(np.float32), idx.astype(np.uint32)


def media_scene(width: int = 1280, height: int = 720, spp: int = 512, max_depth: int = 24, seed: int = 11,
                n_leds: int = 1000, sphere_res=(288, 144), cyl_res=(256, 48), slab_res: int = 24):
    """Many-light and media workload (units: millimetres)."""
    rng = np.random.default_rng(seed)
    scene = Scene()
    # room: floor and back wall
    g = 1500.0
    floor = Lambertian((0.7, 0.7, 0.7))
    fp = np.array([(-g, 0.0, -g), (-g, 0.0, g), (g, 0.0, g), (g, 0.0, -g)], np.float32)
    scene.add_shape(TriangleMesh(fp, None, None, np.array([[0, 1, 2], [0, 2, 3]], np.uint32), floor))
    wall = Lambertian((0.55, 0.55, 0.6))
    wp = np.array([(-g, 0.0, 800.0), (-g, 1200.0, 800.0), (g, 1200.0, 800.0), (g, 0.0, 800.0)], np.float32)
    scene.add_shape(TriangleMesh(wp, None, None, np.array([[0, 1, 2], [0, 2, 3]], np.uint32), wall))
    # LED strip: four seeded colours, each LED quad two triangle emitters
    lpos, lidx = led_strip(n_leds, seed)
    colours = [tuple(rng.uniform(2.0, 8.0) * np.array(c)) for c in ((1.0, 0.85, 0.6), (0.6, 0.8, 1.0), (1.0, 0.5, 0.4),
                                                            (0.7, 1.0, 0.7))]
    which = rng.integers(0, 4, n_leds)
    for k, col in enumerate(colours):
        q = np.nonzero(which == k)[0]
        if q.size == 0:
            continue
        tri = lidx.reshape(2, n_leds, 3)[:, q].reshape(-1, 3)
        used = np.unique(tri)
        remap = np.full(lpos.shape[0], -1, np.int64)
        remap[used] = np.arange(used.size)
        scene.add_shape(TriangleMesh(lpos[used], None, None, remap[tri].astype(np.uint32),
                                     Lambertian((0.0, 0.0, 0.0), emission=col)))
    # dispersive glass sphere
    glass = Dielectric(1.5)
    glass.set_abbe(35.0)
    p, n, i = uv_sphere((-250.0, 95.0, 60.0), 95.0, *sphere_res)
    scene.add_shape(TriangleMesh(p, n, None, i, glass))
    # Henyey–Greenstein scattering sphere (g = 0.6), mean free path ~ 25 mm
    fog = Dielectric(1.33)
    fog.set_scattering(0.04, (0.92, 0.9, 0.85), 0.6)
    p, n, i = uv_sphere((250.0, 95.0, 60.0), 95.0, *sphere_res)
    scene.add_shape(TriangleMesh(p, n, None, i, fog))
    # Beer–Lambert liquid: σa per channel ~ U(0.1, 2) / mm, set as a colour over 1 mm
    sigma_a = rng.uniform(0.1, 2.0, 3)
    liquid = Dielectric(1.33)
    liquid.set_absorption(tuple(np.exp(-sigma_a)), 1.0)
    p, n, i = cylinder((0.0, 0.0, -170.0), 55.0, 110.0, *cyl_res)
    scene.add_shape(TriangleMesh(p, n, None, i, liquid))
    # random-walk subsurface slab, mean free path 1–5 mm per channel
    skin = DisneyMaterial((0.9, 0.62, 0.5), 0.0, 0.45, 0.5)
    skin.set_subsurface(1.0)
    skin.set_subsurface_radius(tuple(rng.uniform(1.0, 5.0, 3)))
    skin.set_subsurface_scale(1.0)
    p, n, i = grid_box((0.0, 20.0, 230.0), (380.0, 40.0, 170.0), slab_res)
    scene.add_shape(TriangleMesh(p, n, None, i, skin))
    camera = camera_for("media", width, height)
    settings = RenderSettings(width=width, height=height, samples_per_pixel=spp, max_bounces=max_depth,
                              filter_type=PixelFilterType.BlackmanHarris, filter_width=1.5)
    return scene, camera, settings


def instanced_grid_scene(width: int = 1920, height: int = 1080, spp: int = 64, max_depth: int = 12, seed: int = 21,
                         nx: int = 5, nz: int = 4, nu: int = 1024, nv: int = 128, env_size=(2048, 1024)):
    """~5M triangles seen: nx·nz rotated, scaled MeshInstances of one knot mesh (one BLAS on the
    device) on a ground plane, each with its own material."""
    rng = np.random.default_rng(seed)
    mats = []
    for _ in range(8):
        m = DisneyMaterial(tuple(rng.uniform(0.0, 1.0, 3)), float(rng.choice([0.0, 1.0])),
                           float(rng.uniform(0.05, 0.9)), 0.5)
        m.set_clear_coat(float(rng.uniform(0.0, 1.0)))
        mats.append(m)
    pos, quads = torus_knot_mesh(nu, nv, seed=seed)
    q = quads.reshape(-1, 4)
    tri = np.concatenate([q[:, [0, 1, 2]], q[:, [0, 2, 3]]], axis=0).astype(np.uint32)
    scene = Scene()
    knot = TriangleMesh(pos.astype(np.float32), None, None, tri, mats[0])
    for i in range(nx):
        for k in range(nz):
            a = rng.uniform(0.0, 2.0 * math.pi)
            sc = rng.uniform(0.6, 0.9)
            c, s_ = math.cos(a), math.sin(a)
            m = np.eye(4)
            m[:3, :3] = np.array([[c, 0.0, s_], [0.0, 1.0, 0.0], [-s_, 0.0, c]]) * sc
            m[:3, 3] = ((i - (nx - 1) / 2) * 5.0, 0.0, (k - (nz - 1) / 2) * 5.0 + 4.0)
            scene.add_shape(MeshInstance(knot, m.astype(np.float32), mats[int(rng.integers(0, 8))]))
    g = 80.0
    gp = np.array([(-g, 0.0, -g), (-g, 0.0, g), (g, 0.0, g), (g, 0.0, -g)], np.float32)
    scene.add_shape(TriangleMesh(gp, None, None, np.array([[0, 1, 2], [0, 2, 3]], np.uint32), Lambertian((0.5, 0.5, 0.5))))
    scene.set_environment(EnvironmentLight(sky_environment(*env_size), 0.0, 1.0))
    settings = RenderSettings(width=width, height=height, samples_per_pixel=spp, max_bounces=max_depth,
                              filter_type=PixelFilterType.BlackmanHarris, filter_width=1.5)
    return scene, camera_for("grid", width, height), settings


def _wall_grid(origin, u, v, nu, nv, hole=None):
    """Quad grid origin + i/nu·u + j/nv·v, facing along u × v; cells whose centre lies in
    hole = (u0, u1, v0, v1) (fractions of u and v) are left open."""
    o, u, v = (np.asarray(a, np.float64) for a in (origin, u, v))
    i, j = np.meshgrid(np.arange(nu + 1), np.arange(nv + 1), indexing="ij")
    pos = o + (i / nu)[..., None] * u + (j / nv)[..., None] * v
    pos = pos.reshape(-1, 3)
    tris = []
    for a in range(nu):
        for b in range(nv):
            if hole is not None:
                cu, cv = (a + 0.5) / nu, (b + 0.5) / nv
                if hole[0] <= cu <= hole[1] and hole[2] <= cv <= hole[3]:
                    continue
            p00 = a * (nv + 1) + b
            p10 = (a + 1) * (nv + 1) + b
            tris.append((p00, p10, p10 + 1))
            tris.append((p00, p10 + 1, p00 + 1))
    return pos.astype(np.float32), np.array(tris, np.uint32)


def room_scene(width: int = 1920, height: int = 1080, spp: int = 64, max_depth: int = 12, seed: int = 5,
               knot_res=(768, 96), env_size=(2048, 1024)):
    """The indirect-lit interior (units: metres)."""
    rng = np.random.default_rng(seed)
    scene = Scene()
    X, Y, Z = 5.0, 3.0, 4.0
    wall = Lambertian((0.75, 0.72, 0.68))
    floor = Lambertian((0.45, 0.33, 0.22))
    ceil = Lambertian((0.85, 0.85, 0.85))
    # inward-facing shell; the window is 1×1 m in the z = −4 wall, 1–2 m above the floor
    for (o, u, v, nu, nv, hole, mat) in (
            ((-X, 0.0, -Z), (2 * X, 0.0, 0.0), (0.0, Y, 0.0), 100, 30, (0.45, 0.55, 1 / 3, 2 / 3), wall),  # z = −4 (window)
            ((X, 0.0, Z), (-2 * X, 0.0, 0.0), (0.0, Y, 0.0), 100, 30, None, wall),                         # z = +4
            ((-X, 0.0, Z), (0.0, 0.0, -2 * Z), (0.0, Y, 0.0), 80, 30, None, wall),                          # x = −5
            ((X, 0.0, -Z), (0.0, 0.0, 2 * Z), (0.0, Y, 0.0), 80, 30, None, wall),                           # x = +5
            ((-X, 0.0, Z), (2 * X, 0.0, 0.0), (0.0, 0.0, -2 * Z), 100, 80, None, floor),                   # floor
            ((-X, Y, -Z), (2 * X, 0.0, 0.0), (0.0, 0.0, 2 * Z), 100, 80, None, ceil)):                     # ceiling
        pos, idx = _wall_grid(o, u, v, nu, nv, hole)
        scene.add_shape(TriangleMesh(pos, None, None, idx, mat))
    # furniture: three knots, a sphere, two tables
    pos, quads = torus_knot_mesh(*knot_res, tube=0.38, seed=seed)
    q = quads.reshape(-1, 4)
    tri = np.concatenate([q[:, [0, 1, 2]], q[:, [0, 2, 3]]], axis=0).astype(np.uint32)
    for k, (cx, cz, sc) in enumerate(((-2.5, -1.0, 0.45), (1.5, -2.0, 0.4), (0.0, 1.5, 0.5))):
        m = DisneyMaterial(tuple(rng.uniform(0.2, 0.9, 3)), 0.0 if k != 1 else 1.0, float(rng.uniform(0.2, 0.6)), 0.5)
        a = rng.uniform(0.0, 2.0 * math.pi)
        c, s_ = math.cos(a), math.sin(a)
        rot = np.array([[c, 0.0, s_], [0.0, 1.0, 0.0], [-s_, 0.0, c]])
        p = (pos @ rot.T) * sc + np.array([cx, 1.0 * sc + 0.45, cz])
        scene.add_shape(TriangleMesh(p.astype(np.float32), None, None, tri, m))
    p, n, i = uv_sphere((3.0, 0.6, -1.0), 0.6, 256, 128)
    scene.add_shape(TriangleMesh(p, n, None, i, DisneyMaterial((0.8, 0.8, 0.85), 0.0, 0.15, 0.5)))
    table = Lambertian((0.5, 0.4, 0.3))
    for (tx, tz) in ((-2.5, 2.5), (2.5, 2.0)):
        pb, ib, = _box((tx, 0.4, tz), (1.6, 0.8, 1.0), 10.0)
        scene.add_shape(TriangleMesh(pb, None, None, ib, table))
    scene.set_environment(EnvironmentLight(sky_environment(*env_size), 0.0, 1.0))
    settings = RenderSettings(width=width, height=height, samples_per_pixel=spp, max_bounces=max_depth,
                              filter_type=PixelFilterType.BlackmanHarris, filter_width=1.5)
    return scene, camera_for("room", width, height), settings
