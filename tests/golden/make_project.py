"""Writes tests/golden/studio.photon: a small project in the photon engine's project format
(JSON, "photon-project" version 2) whose content is this repository's own — a transformed group
with a box mesh and an octahedron mesh, spheres under a scaling transform, Disney / glass / mirror /
Lambert materials with advanced keys, an area light, the automatic ground quad and the procedural
studio sky — used to check the .photon loader against the reference's loader.

    python tests/golden/make_project.py
"""
import json
import math
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def box(size):
    sx, sy, sz = (s * 0.5 for s in size)
    p, i = [], []
    faces = [((1, 0, 0), (0, 1, 0), (0, 0, 1)), ((-1, 0, 0), (0, 0, 1), (0, 1, 0)), ((0, 1, 0), (0, 0, 1), (1, 0, 0)),
             ((0, -1, 0), (1, 0, 0), (0, 0, 1)), ((0, 0, 1), (1, 0, 0), (0, 1, 0)), ((0, 0, -1), (0, 1, 0), (1, 0, 0))]
    for n, u, v in faces:
        c = np.array(n, float) * (sx, sy, sz)
        du = np.array(u, float) * (sx, sy, sz)
        dv = np.array(v, float) * (sx, sy, sz)
        base = len(p)
        for a, b in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
            p.append(c + a * du + b * dv)
        i += [base, base + 1, base + 2, base, base + 2, base + 3]
    return np.array(p), np.array(i)


def knot(nu=96, nv=12, r=0.12):
    t = np.linspace(0, 2 * math.pi, nu, endpoint=False)
    c = np.stack([(np.cos(3 * t) + 2) * np.cos(2 * t), -np.sin(3 * t), (np.cos(3 * t) + 2) * np.sin(2 * t)], -1) * 0.18
    tang = np.roll(c, -1, 0) - np.roll(c, 1, 0)
    tang /= np.linalg.norm(tang, axis=1, keepdims=True)
    n = np.cross(tang, [0.0, 1.0, 0.0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    b = np.cross(tang, n)
    a = np.linspace(0, 2 * math.pi, nv, endpoint=False)
    p = c[:, None] + r * (np.cos(a)[None, :, None] * n[:, None] + np.sin(a)[None, :, None] * b[:, None])
    idx = []
    for k in range(nu):
        for j in range(nv):
            q = [k * nv + j, ((k + 1) % nu) * nv + j, ((k + 1) % nu) * nv + (j + 1) % nv, k * nv + (j + 1) % nv]
            idx += [q[0], q[1], q[2], q[0], q[2], q[3]]
    return p.reshape(-1, 3), np.array(idx)


def octahedron(r=0.3):
    p = np.array([(r, 0, 0), (-r, 0, 0), (0, r, 0), (0, -r, 0), (0, 0, r), (0, 0, -r)], float)
    i = [0, 2, 4, 2, 1, 4, 1, 3, 4, 3, 0, 4, 2, 0, 5, 1, 2, 5, 3, 1, 5, 0, 3, 5]
    return p, np.array(i)


def xf_trs(t=(0, 0, 0), ry_deg=0.0, s=1.0):
    c, si = math.cos(math.radians(ry_deg)), math.sin(math.radians(ry_deg))
    return [s * c, 0, s * si, t[0], 0, s, 0, t[1], -s * si, 0, s * c, t[2], 0, 0, 0, 1]


def mesh_node(name, mat, p, i, xf):
    return {"type": "mesh", "name": name, "visible": True, "material": mat, "xf": xf,
            "geometry": {"p": [round(float(x), 6) for x in p.ravel()], "i": [int(k) for k in i]}}


def main():
    # meshes of at most 16 triangles: the reference intersects those without a BLAS traversal
    # (larger instanced meshes meet its shared-stack defect, checked separately)
    bp, bi = box((0.5, 0.7, 0.5))
    kp, ki = octahedron()
    materials = [
        {"type": "disney", "baseColor": [0.8, 0.35, 0.2], "metallic": 0.0, "roughness": 0.4, "specular": 0.5,
         "clearCoat": 0.6, "clearCoatRoughness": 0.1, "sheenColor": [0.9, 0.8, 0.7], "sheen": 0.3},
        {"type": "disney", "baseColor": [0.9, 0.85, 0.8], "metallic": 1.0, "roughness": 0.25, "edgeTint": [0.9, 0.7, 0.5]},
        {"type": "glass", "ior": 1.45, "tint": [0.95, 0.98, 1.0], "roughness": 0.0},
        {"type": "mirror", "color": [0.92, 0.92, 0.92]},
        {"type": "lambert", "albedo": [0.3, 0.5, 0.7], "emission": [0, 0, 0]},
    ]
    nodes = [
        {"type": "group", "name": "table", "visible": True, "xf": xf_trs((0.2, 0.0, -0.1), 25.0),
         "children": [mesh_node("box", 0, bp + (0, 0.35, 0), bi, xf_trs((-0.5, 0, 0), 10.0)),
                      mesh_node("gem", 1, kp + (0, 0.6, 0), ki, xf_trs((0.45, 0, 0.1), -30.0, 0.9))]},
        {"type": "group", "name": "spheres", "visible": True, "xf": xf_trs((0.0, 0.0, 0.5), 0.0, 1.2),
         "children": [{"type": "sphere", "name": "glass", "visible": True, "material": 2, "radius": 0.25,
                       "xf": xf_trs((-0.2, 0.25, 0.2))},
                      {"type": "sphere", "name": "mirror", "visible": True, "material": 3, "radius": 0.18,
                       "xf": xf_trs((0.35, 0.18, 0.25))},
                      {"type": "sphere", "name": "hidden", "visible": False, "material": 4, "radius": 0.3,
                       "xf": xf_trs((0.0, 1.0, 0.0))}]},
        {"type": "sphere", "name": "blue", "visible": True, "material": 4, "radius": 0.2, "xf": xf_trs((-0.8, 0.2, 0.6))},
    ]
    project = {
        "format": "photon-project", "version": 2,
        "camera": {"target": [0.0, 0.45, 0.1], "radius": 3.2, "theta": 1.2, "phi": 1.1, "fov": 38.0, "aperture": 0.0,
                   "orthographic": False},
        "environment": {"hdr": "", "zenith": [0.55, 0.65, 0.9], "horizon": [0.6, 0.58, 0.55], "rotation": 30.0,
                        "intensity": 0.8, "background": {"mode": "environment", "color": [0, 0, 0]},
                        "ground": {"enabled": True, "color": [0.45, 0.43, 0.4], "roughness": 0.6,
                                   "shadowCatcher": False}},
        "lights": [{"type": "area", "name": "key", "enabled": True, "color": [1.0, 0.95, 0.9], "intensity": 6.0,
                    "position": [1.5, 2.2, 1.2], "target": [0.0, 0.3, 0.0], "width": 0.8, "height": 0.5,
                    "visibleToCamera": True}],
        "materials": materials,
        "nodes": nodes,
        "render": {"maxBounces": 6, "pixelFilter": "gaussian", "filterWidth": 1.5},
    }
    (HERE / "studio.photon").write_text(json.dumps(project, indent=1))


if __name__ == "__main__":
    main()
