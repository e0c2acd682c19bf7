"""Seeded procedural workload descriptions as plain numpy data (no engine, no library load).

A description is a dict that either side of a comparison can turn into a scene: the product's
``scenes.from_description`` builds ``engine.Scene`` objects from it, and the reference's CPU path
can be fed the same arrays without the product library being loaded.

Layout::

    {"materials":   [{"type": 0|1|2|3, <pe_material field>: value, ...}, ...],
     "ops":         [("mesh", {"positions", "indices", "material", "normals"?, "uvs"?}),
                     ("area", {"position", "u", "v", "radiance"}), ...],
     "environment": {"image", "rotation", "intensity"} or None,
     "camera":      {"position", "target", "up", "vfov", "aspect"},
     "settings":    RenderSettings fields}

Material dicts name ``pe_material`` fields (``include/photon_cuda.h``); fields left out keep
``pe_material_defaults``.  ``type`` is PE_MAT_LAMBERT (0), PE_MAT_DISNEY (1), PE_MAT_DIELECTRIC (2)
or PE_MAT_MIRROR (3).
"""
from __future__ import annotations

import numpy as np

MAT_LAMBERT, MAT_DISNEY, MAT_DIELECTRIC, MAT_MIRROR = range(4)
FILTER_BLACKMAN_HARRIS = 3

# Viewpoints of the workloads: (position, target, up, vertical fov in degrees).
CAMERAS = {
    "cornell": ((2.78, 2.73, -8.0), (2.78, 2.73, 0.0), (0.0, 1.0, 0.0), 39.3),
    "knot": ((0.0, 4.5, -10.5), (0.0, 1.6, 0.0), (0.0, 1.0, 0.0), 40.0),
    "media": ((0.0, 420.0, -950.0), (0.0, 70.0, 40.0), (0.0, 1.0, 0.0), 38.0),
    "grid": ((0.0, 8.0, -13.0), (0.0, 1.0, 4.0), (0.0, 1.0, 0.0), 45.0),
    "room": ((4.2, 1.7, 3.4), (-1.5, 0.9, -2.5), (0.0, 1.0, 0.0), 62.0),
}


def camera_desc(name: str, width: int, height: int) -> dict:
    pos, target, up, fov = CAMERAS[name]
    return {"position": pos, "target": target, "up": up, "vfov": fov, "aspect": width / height}


def _knot_curve(t, p=2, q=3):
    r = np.cos(q * t) + 2.0
    return np.stack([r * np.cos(p * t), -np.sin(q * t), r * np.sin(p * t)], axis=-1)


def knot_mesh(nu: int = 4096, nv: int = 128, tube: float = 0.38, seed: int = 1):
    """(2,3) torus knot tube with nu × nv quads (2·nu·nv triangles), seeded radial jitter.
    Returns float32 positions (nu·nv, 3) and the quads' vertex indices (nu, nv, 4)."""
    rng = np.random.default_rng(seed)
    t = np.linspace(0.0, 2.0 * np.pi, nu, endpoint=False)
    c = _knot_curve(t)
    dt = 1e-3
    tangent = _knot_curve(t + dt) - _knot_curve(t - dt)
    tangent /= np.linalg.norm(tangent, axis=1, keepdims=True)
    # rotation-minimising frame by parallel transport
    nrm = np.empty_like(tangent)
    ref = np.array([0.0, 1.0, 0.0])
    n0 = np.cross(tangent[0], ref)
    nrm[0] = n0 / np.linalg.norm(n0)
    for i in range(1, nu):
        n = nrm[i - 1] - tangent[i] * np.dot(nrm[i - 1], tangent[i])
        nrm[i] = n / np.linalg.norm(n)
    binrm = np.cross(tangent, nrm)
    ang = np.linspace(0.0, 2.0 * np.pi, nv, endpoint=False)
    radius = tube * (1.0 + 0.02 * rng.standard_normal((nu, nv)))
    pos = (c[:, None, :] + radius[..., None] * (np.cos(ang)[None, :, None] * nrm[:, None, :] +
                                                np.sin(ang)[None, :, None] * binrm[:, None, :]))
    pos = (pos + np.array([0.0, 1.9, 0.0])).astype(np.float32).reshape(-1, 3)
    i = np.arange(nu)[:, None]
    j = np.arange(nv)[None, :]
    a = i * nv + j
    b = ((i + 1) % nu) * nv + j
    cc = ((i + 1) % nu) * nv + (j + 1) % nv
    d = i * nv + (j + 1) % nv
    quads = np.stack([a, b, cc, d], axis=-1).reshape(nu, nv, 4)
    return pos, quads


def sky_image(width: int = 2048, height: int = 1024, sun_dir=(0.45, 0.62, -0.64), sun_share: float = 0.6,
              sun_sigma_deg: float = 1.5, seed: int = 2) -> np.ndarray:
    """Sky gradient plus one Gaussian sun lobe holding ``sun_share`` of the (solid-angle weighted)
    luminance, in the reference's equirect convention (v = θ/π, y up, φ = atan2(−z, x) + π)."""
    rng = np.random.default_rng(seed)
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    theta = v * np.pi
    a = u * 2.0 * np.pi - np.pi
    st = np.sin(theta)[:, None]
    d = np.stack([st * np.cos(a)[None, :], np.cos(theta)[:, None] * np.ones((1, width)), -st * np.sin(a)[None, :]], -1)
    up = d[..., 1]
    zenith = np.array([0.25, 0.45, 1.0])
    horizon = np.array([1.0, 0.95, 0.9])
    ground = np.array([0.18, 0.16, 0.14])
    tsky = np.clip(up, 0.0, 1.0)[..., None]
    sky = np.where(up[..., None] >= 0.0, horizon * (1 - tsky) + zenith * tsky, ground)
    sky = sky * (1.0 + 0.02 * rng.standard_normal((height, width, 1)))
    sdir = np.asarray(sun_dir, np.float64)
    sdir /= np.linalg.norm(sdir)
    cosang = np.clip((d * sdir).sum(-1), -1.0, 1.0)
    ang = np.arccos(cosang)
    lobe = np.exp(-0.5 * (ang / np.radians(sun_sigma_deg)) ** 2)
    w = np.sin(theta)[:, None]
    lum = lambda img: (0.212671 * img[..., 0] + 0.715160 * img[..., 1] + 0.072169 * img[..., 2])
    sky_power = float((lum(sky) * w).sum())
    lobe_power = float((lobe * w).sum())
    k = sun_share / (1.0 - sun_share) * sky_power / lobe_power
    sun_color = np.array([1.0, 0.93, 0.8])
    img = sky + k * lobe[..., None] * sun_color / lum(sun_color[None, None, :])[..., None]
    return img.astype(np.float32)


def torus_knot(width: int = 1920, height: int = 1080, spp: int = 256, max_depth: int = 12, nu: int = 4096,
               nv: int = 128, env_size=(2048, 1024), seed: int = 7, clusters: int = 64) -> dict:
    """Product-scale workload: ~1M-triangle torus knot whose random face clusters carry eight
    Disney materials (metallic ∈ {0,1}, roughness ~ U(0.05, 0.9), clearcoat ~ U(0,1), base
    ~ U(0,1)³), a ground plane, a float32 sky whose sun lobe holds 60 % of the power, one
    rectangular softbox."""
    rng = np.random.default_rng(seed)
    mats = []
    for _ in range(8):
        base = tuple(float(x) for x in rng.uniform(0.0, 1.0, 3))
        metallic = float(rng.choice([0.0, 1.0]))
        roughness = float(rng.uniform(0.05, 0.9))
        mats.append({"type": MAT_DISNEY, "base_color": base, "metallic": metallic, "roughness": roughness,
                     "specular": 0.5, "clearcoat": float(rng.uniform(0.0, 1.0))})
    mats.append({"type": MAT_LAMBERT, "base_color": (0.5, 0.5, 0.5)})
    ops = []
    pos, quads = knot_mesh(nu, nv, seed=seed)
    # random face clusters: contiguous runs of rings along the knot, each with one material
    cuts = np.sort(rng.choice(np.arange(1, nu), clusters - 1, replace=False))
    bounds = np.concatenate([[0], cuts, [nu]])
    for k in range(clusters):
        q = quads[bounds[k]:bounds[k + 1]].reshape(-1, 4)
        tri = np.concatenate([q[:, [0, 1, 2]], q[:, [0, 2, 3]]], axis=0)
        used = np.unique(tri)
        remap = np.full(pos.shape[0], -1, np.int64)
        remap[used] = np.arange(used.size)
        ops.append(("mesh", {"positions": pos[used], "indices": remap[tri].astype(np.uint32),
                             "material": int(rng.integers(0, 8))}))
    g = 40.0
    gp = np.array([(-g, 0.0, -g), (-g, 0.0, g), (g, 0.0, g), (g, 0.0, -g)], np.float32)
    ops.append(("mesh", {"positions": gp, "indices": np.array([[0, 1, 2], [0, 2, 3]], np.uint32), "material": 8}))
    ops.append(("area", {"position": (-3.0, 6.5, -2.0), "u": (3.0, 0.0, 0.0), "v": (0.0, 0.0, 2.0),
                         "radiance": (12.0, 12.0, 12.0)}))
    return {"materials": mats, "ops": ops,
            "environment": {"image": sky_image(*env_size), "rotation": 0.0, "intensity": 1.0},
            "camera": camera_desc("knot", width, height),
            "settings": {"width": width, "height": height, "samples_per_pixel": spp, "max_bounces": max_depth,
                         "filter_type": FILTER_BLACKMAN_HARRIS, "filter_width": 1.5}}


def triangle_count(desc: dict) -> int:
    """Triangles of a description (each area light adds its two)."""
    return sum(int(o["indices"].shape[0]) if kind == "mesh" else 2 for kind, o in desc["ops"])
