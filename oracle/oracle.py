"""TEST INFRASTRUCTURE (oracle) — not part of the product.

ctypes driver of the reference engine's own CPU path (``_ref/libphoton_ref.so``, built from the
reference sources by ``oracle/Makefile``) and of the C restatement (``_ref/libpe_oracle.so``).
Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this module, and
only as the checker / the timed CPU baseline.

``RefScene(scene)`` replays a product ``Scene`` (its recorded ``ops``, environment and
background) through the reference's Scene API in the same order, so both sides hold the same
shapes, lights, light indices and BVH input order.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
PARITY_LIB = REF_DIR / "libphoton_ref.so"
FAST_LIB = REF_DIR / "libphoton_ref_fast.so"
RESTATEMENT_LIB = REF_DIR / "libpe_oracle.so"
ADAPTER_LIB = REF_DIR / "libpe_adapter.so"  # the reference engine + the drop-in adapter over libphoton_cuda.so

FP = C.POINTER(C.c_float)
IP = C.POINTER(C.c_int32)
UP = C.POINTER(C.c_uint32)

_libs: dict = {}


def available(fast: bool = False) -> bool:
    return (FAST_LIB if fast else PARITY_LIB).exists()


def adapter_available() -> bool:
    return ADAPTER_LIB.exists()


def _load(fast=False):
    """fast: False the parity build, True the shipping build, "adapter" the parity build linked
    with the drop-in RenderDevice adapter."""
    key = "adapter" if fast == "adapter" else ("fast" if fast else "parity")
    if key in _libs:
        return _libs[key]
    path = ADAPTER_LIB if key == "adapter" else (FAST_LIB if fast else PARITY_LIB)
    if not path.exists():
        raise RuntimeError(f"{path} missing: build it with `make -C oracle` where the reference sources exist")
    lib = C.CDLL(str(path))
    P = C.c_void_p
    sig = {
        "ref_scene_create": (P, []),
        "ref_scene_destroy": (None, [P]),
        "ref_scene_add_material": (C.c_int32, [P, C.c_void_p]),
        "ref_scene_add_mesh": (C.c_int32, [P, FP, C.c_uint32, FP, FP, UP, C.c_uint32, C.c_int32]),
        "ref_scene_add_area_light": (C.c_int32, [P, FP, FP, FP, FP, C.c_int32]),
        "ref_scene_set_environment": (C.c_int32, [P, FP, C.c_int32, C.c_int32, C.c_float, C.c_float, FP, C.c_float, FP]),
        "ref_scene_set_background": (C.c_int32, [P, C.c_int32, FP]),
        "ref_scene_build": (C.c_int32, [P]),
        "ref_scene_light_count": (C.c_int32, [P]),
        "ref_scene_light_mode": (C.c_int32, [P]),
        "ref_camera_perspective": (None, [FP, FP, FP, C.c_float, C.c_float, C.c_void_p]),
        "ref_render": (C.c_int32, [P, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, FP, UP]),
        "ref_render_seeded": (C.c_int32, [P, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, FP, UP]),
"ref_render_rows": (C.c_int32, [P, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                            C.c_int32, FP, UP]),
        "ref_trace_primary": (C.c_int32, [P, C.c_void_p, C.c_void_p, C.c_int32, IP, IP, FP]),
        "ref_sobol": (C.c_int32, [C.c_uint64, IP, IP, IP, C.c_size_t, C.c_int32, FP]),
        "ref_sobol_1d": (C.c_int32, [C.c_uint64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, FP]),
        "ref_bsdf_probe": (C.c_int32, [P, C.c_int32, C.c_void_p, C.c_size_t, C.c_void_p]),
        "ref_light_pick": (C.c_int32, [P, FP, FP, FP, C.c_size_t, IP, FP, FP]),
        "ref_light_sample": (C.c_int32, [P, C.c_int32, FP, FP, FP, C.c_size_t, FP, FP, FP, FP]),
        "ref_env_eval": (C.c_int32, [P, FP, C.c_size_t, FP, FP]),
        "ref_render_guided": (C.c_int32, [P, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, FP, UP]),
        "ref_scene_set_shadow_catcher": (C.c_int32, [P, C.c_int32]),
        "ref_scene_set_light_group": (C.c_int32, [P, C.c_int32, C.c_char_p]),
        "ref_scene_add_texture": (C.c_int32, [P, FP, C.c_int32, C.c_int32]),
        "ref_render_crypto": (C.c_int32, [P, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, FP, C.c_int32]),
        "ref_scene_set_shape_name": (C.c_int32, [P, C.c_int32, C.c_char_p]),
        "ref_scene_set_shape_visibility": (C.c_int32, [P, C.c_int32, C.c_uint32]),
        "ref_scene_set_material_name": (C.c_int32, [P, C.c_int32, C.c_char_p]),
        "ref_scene_build_texture_mipmaps": (C.c_int32, [P, C.c_int32]),
        "ref_scene_add_texture_u8": (C.c_int32, [P, C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
        "ref_film_create": (P, [C.c_int32, C.c_int32]),
        "ref_film_destroy": (None, [P]),
        "ref_film_export": (C.c_int32, [P, C.c_int32, C.c_int32, FP, UP]),
        "ref_render_film": (C.c_int64, [P, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, P]),
        "ref_render_passes": (C.c_int32, [P, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, FP, UP, FP, FP,
                                          FP, C.c_int32]),
        "ref_render_aovs": (C.c_int32, [P, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, FP, UP, FP, FP,
                                        FP, UP]),
        "ref_scene_tag_shape": (C.c_int32, [P, C.c_int32, C.c_uint64]),
        "ref_scene_set_light_link": (C.c_int32, [P, C.c_int32, C.c_int32, C.POINTER(C.c_uint64), C.c_int32,
                                                 C.c_int32, C.POINTER(C.c_uint64), C.c_int32]),
        "ref_camera_create": (P, [C.c_int32, FP]),
        "ref_camera_destroy": (None, [P]),
        "ref_camera_describe": (None, [P, C.c_void_p]),
        "ref_render_rows_camera": (C.c_int32, [P, P, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                               C.c_int32, FP, UP]),
        "ref_dtree_probe": (C.c_int32, [FP, FP, C.c_int32, FP, FP, C.c_int32, FP, FP, C.c_int32, FP, FP]),
        "ref_render_camera": (C.c_int32, [P, P, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, FP, UP]),
        "ref_scene_add_sphere": (C.c_int32, [P, FP, C.c_float, C.c_int32]),
        "ref_scene_add_blas": (C.c_int32, [P, FP, C.c_uint32, FP, FP, UP, C.c_uint32]),
        "ref_scene_add_instance": (C.c_int32, [P, C.c_int32, FP, FP, C.c_int32]),
        "ref_scene_move_instance": (C.c_int32, [P, C.c_int32, FP, FP]),
        "ref_scene_set_instance_motion": (C.c_int32, [P, C.c_int32, FP, FP]),
        "ref_scene_shape_count": (C.c_int32, [P]),
        "ref_trace_rays": (C.c_int32, [P, FP, FP, FP, C.c_int32, C.c_int32, C.c_uint32, C.c_float, IP, IP, FP]),
        "ref_camera_set_shutter_end": (None, [P, P]),
        "ref_load_project": (P, [C.c_char_p, C.c_float, IP, FP, IP, IP, FP, C.c_char_p, C.c_size_t]),
        "ref_scene_shapes": (C.c_int32, [P, IP, IP, FP, C.c_int32]),
        "ref_material_defaults": (None, [C.c_int32, C.c_void_p]),
        "ref_render_rect": (C.c_int32, [P, P, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                        C.c_int32, C.c_int32, FP, UP]),
    }
    if key == "adapter":
        sig["ref_session_cuda"] = (C.c_int32, [P, P, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, FP, UP, FP,
                                               IP, C.c_char_p, C.c_size_t])
        sig["ref_session_cuda_update"] = (C.c_int32, [P, C.c_int32, C.c_int32, FP])
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _libs[key] = lib
    return lib


def _f(a):
    return None if a is None else a.ctypes.data_as(FP)


def _f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


class RefFilm:
    """A reference Film kept across render calls."""

    def __init__(self, width: int, height: int, fast: bool = False):
        self.lib = _load(fast)
        self.width, self.height = width, height
        self.h = self.lib.ref_film_create(width, height)

    def __del__(self):
        try:
            self.lib.ref_film_destroy(self.h)
        except Exception:
            pass

    def mean_and_counts(self):
        mean = np.zeros((self.height, self.width, 3), np.float32)
        cnt = np.zeros((self.height, self.width), np.uint32)
        self.lib.ref_film_export(self.h, self.width, self.height, _f(mean), cnt.ctypes.data_as(UP))
        return mean, cnt


class RefScene:
    """The reference engine's Scene holding the same content as a product Scene."""

    def __init__(self, scene, fast: bool = False):
        self.lib = _load(fast)
        self.h = self.lib.ref_scene_create()
        tex_index = {}
        for img in (scene.textures() if hasattr(scene, "textures") else []):
            if img.dtype == np.uint8:
                srgb = not any(id(img) in getattr(m, "linear_u8", ()) for m in scene.materials())
                tex_index[id(img)] = self.lib.ref_scene_add_texture_u8(self.h, img.ctypes.data, img.shape[1],
                                                                       img.shape[0], 1 if srgb else 0)
            else:
                tex_index[id(img)] = self.lib.ref_scene_add_texture(self.h, _f(img), img.shape[1], img.shape[0])
            if scene.texture_has_mipmaps(img):
                self.lib.ref_scene_build_texture_mipmaps(self.h, tex_index[id(img)])
        mat_index = {}
        for kind, obj in scene.ops:
            if kind in ("mesh", "sphere", "instance") and id(obj.material) not in mat_index:
                struct = obj.material.struct_with(tex_index) if hasattr(obj.material, "struct_with") \
                    else obj.material.struct
                idx = self.lib.ref_scene_add_material(self.h, C.byref(struct))
                if idx < 0:
                    raise RuntimeError("reference rejected a material")
                mat_index[id(obj.material)] = idx
        self.mat_index = mat_index
        blas_index = {}
        for kind, obj in scene.ops:
            if kind == "sphere":
                rc = self.lib.ref_scene_add_sphere(self.h, _f3(obj.center), obj.radius, mat_index[id(obj.material)])
            elif kind == "instance":
                mesh = obj.mesh
                if id(mesh) not in blas_index:
                    blas_index[id(mesh)] = self.lib.ref_scene_add_blas(
                        self.h, _f(mesh.positions), mesh.positions.shape[0], _f(mesh.normals), _f(mesh.uvs),
                        mesh.indices.ctypes.data_as(UP), mesh.indices.shape[0])
                rc = self.lib.ref_scene_add_instance(self.h, blas_index[id(mesh)], _f(obj.local_to_world),
                                                     _f(obj.world_to_local), mat_index[id(obj.material)])
                if rc == 0 and getattr(obj, "local_to_world_end", None) is not None:
                    rc = self.lib.ref_scene_set_instance_motion(self.h, self.lib.ref_scene_shape_count(self.h) - 1,
                                                                _f(obj.local_to_world_end), _f(obj.world_to_local_end))
            elif kind == "mesh":
                rc = self.lib.ref_scene_add_mesh(self.h, _f(obj.positions), obj.positions.shape[0], _f(obj.normals),
                                                 _f(obj.uvs), obj.indices.ctypes.data_as(UP), obj.indices.shape[0],
                                                 mat_index[id(obj.material)])
            else:
                rc = self.lib.ref_scene_add_area_light(self.h, _f3(obj.position), _f3(obj.u), _f3(obj.v),
                                                       _f3(obj.radiance), 1 if obj.visible_to_camera else 0)
            if rc != 0:
                raise RuntimeError("reference rejected a shape")
        if getattr(scene, "shadow_catcher", None) is not None:
            self.lib.ref_scene_set_shadow_catcher(self.h, int(scene.shadow_catcher))
        for shape, uid in getattr(scene, "shape_tags", {}).items():
            if self.lib.ref_scene_tag_shape(self.h, int(shape), int(uid)) != 0:
                raise RuntimeError("reference rejected a shape tag")
        for shape, name in getattr(scene, "shape_names", {}).items():
            self.lib.ref_scene_set_shape_name(self.h, int(shape), name.encode())
        shape = 0
        for kind, obj in scene.ops:
            if kind != "area" and getattr(obj, "visibility_mask", 0x1F) != 0x1F:
                self.lib.ref_scene_set_shape_visibility(self.h, shape, int(obj.visibility_mask))
            shape += 2 if kind == "area" else 1
        for mat, name in getattr(scene, "material_names", {}).values():
            if id(mat) in mat_index:
                self.lib.ref_scene_set_material_name(self.h, mat_index[id(mat)], name.encode())
        for light, (mode, uids, smode, suids) in getattr(scene, "light_links", {}).items():
            a = (C.c_uint64 * max(1, len(uids)))(*uids)
            b = (C.c_uint64 * max(1, len(suids)))(*suids)
            if self.lib.ref_scene_set_light_link(self.h, int(light), int(mode), a, len(uids), int(smode), b,
                                                 len(suids)) != 0:
                raise RuntimeError("reference rejected a light link")
        # light groups: an area light's own, then Scene.set_light_group's (light numbering as in
        # the product scene: one per area light, one per triangle of an emissive mesh)
        groups, li = {}, 0
        for kind, obj in scene.ops:
            if kind == "sphere":
                continue
            if kind in ("mesh", "instance"):
                m = obj.material.struct
                if m.type in (0, 1) and any(m.emission):
                    li += (obj.mesh if kind == "instance" else obj).indices.shape[0]
            else:
                if getattr(obj, "light_group", ""):
                    groups[li] = obj.light_group
                li += 1
        groups.update(getattr(scene, "light_groups", {}))
        for light, name in groups.items():
            if self.lib.ref_scene_set_light_group(self.h, int(light), name.encode()) != 0:
                raise RuntimeError("reference rejected a light group")
        env = scene.environment
        if env is not None and getattr(env, "light_group", ""):
            self.lib.ref_scene_set_light_group(self.h, -1, env.light_group.encode())
        if env is not None:
            img = env.image
            sun = env.sun
            self.lib.ref_scene_set_environment(self.h, _f(img), 0 if img is None else img.shape[1],
                                               0 if img is None else img.shape[0], env.rotation, env.intensity,
                                               _f3(sun[0]) if sun else None, sun[1] if sun else 1.0,
                                               _f3(sun[2]) if sun else None)
        self.lib.ref_scene_set_background(self.h, int(scene.background.mode), _f3(scene.background.color))
        self.lib.ref_scene_build(self.h)

    def __del__(self):
        try:
            self.lib.ref_scene_destroy(self.h)
        except Exception:
            pass

    def light_count(self) -> int:
        return self.lib.ref_scene_light_count(self.h)

    def light_mode(self) -> int:
        return self.lib.ref_scene_light_mode(self.h)

    def render(self, camera, settings, first: int, count: int, threads: int = 0, seeded: bool = True):
        """Mean image (h, w, 3) and counts of samples [first, first+count).  ``seeded`` runs the
        tracePixel loop with settings.seed; otherwise Renderer::renderSamples (seed 12345).  A
        thin-lens or orthographic camera renders through the reference's own camera class."""
        h, w = settings.height, settings.width
        mean = np.zeros((h, w, 3), np.float32)
        cnt = np.zeros((h, w), np.uint32)
        kind = camera.reference_params()[0] if hasattr(camera, "reference_params") else 0
        if kind != 0 and seeded:
            cam = reference_camera(camera, self.lib)
            try:
                self.lib.ref_render_rows_camera(self.h, cam, C.byref(settings.to_c()), first, count, threads, 0, h,
                                                _f(mean), cnt.ctypes.data_as(UP))
            finally:
                self.lib.ref_camera_destroy(cam)
            return mean, cnt
        fn = self.lib.ref_render_seeded if seeded else self.lib.ref_render
        fn(self.h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()), first, count, threads, _f(mean),
           cnt.ctypes.data_as(UP))
        return mean, cnt

    def render_rect(self, camera, settings, rect, first: int, count: int, threads: int = 0):
        """Mean (h, w, 3) and counts of samples [first, first+count) of the pixels of
        rect = (x0, y0, w, h) of the frame: the seeded tracePixel loop through the reference's own
        camera class."""
        x0, y0, w, h = (int(v) for v in rect)
        mean = np.zeros((h, w, 3), np.float32)
        cnt = np.zeros((h, w), np.uint32)
        cam = reference_camera(camera, self.lib)
        try:
            rc = self.lib.ref_render_rect(self.h, cam, C.byref(settings.to_c()), first, count, threads, x0, y0, w, h,
                                          _f(mean), cnt.ctypes.data_as(UP))
        finally:
            self.lib.ref_camera_destroy(cam)
        if rc != 0:
            raise ValueError(f"rectangle {rect} outside the {settings.width}x{settings.height} frame")
        return mean, cnt

    def session_cuda(self, camera, settings, spp: int, batch: int = 8, aovs: bool = False, adaptive: bool = False):
        """RenderSession (begin, advance until finished) on the B200 device through the drop-in
        RenderDevice adapter (RefScene built with fast="adapter").  Returns (mean, counts,
        albedo mean or None, samples per pixel done, features bits: 1 aovs, 2 lightPasses, 4
        adaptiveSampling)."""
        h, w = settings.height, settings.width
        mean = np.zeros((h, w, 3), np.float32)
        cnt = np.zeros((h, w), np.uint32)
        alb = np.zeros((h, w, 3), np.float32) if aovs else None
        feats = C.c_int32(0)
        err = C.create_string_buffer(512)
        cam = reference_camera(camera, self.lib)
        try:
            done = self.lib.ref_session_cuda(self.h, cam, C.byref(settings.to_c()), spp, batch, 1 if aovs else 0,
                                             1 if adaptive else 0, _f(mean), cnt.ctypes.data_as(UP), _f(alb),
                                             C.byref(feats), err, len(err))
        finally:
            self.lib.ref_camera_destroy(cam)
        if done < 0:
            raise RuntimeError(f"adapter session failed ({done}): {err.value.decode()}")
        return mean, cnt, alb, int(done), int(feats.value)

    def move_instance(self, shape: int, local_to_world, world_to_local=None):
        """Places MeshInstance `shape` anew with another matrix (same mesh and material) and
        rebuilds the reference scene's accelerator."""
        m = np.ascontiguousarray(local_to_world, np.float32).reshape(16)
        mi = None if world_to_local is None else np.ascontiguousarray(world_to_local, np.float32).reshape(16)
        if self.lib.ref_scene_move_instance(self.h, int(shape), _f(m), None if mi is None else _f(mi)) != 0:
            raise ValueError(f"shape {shape} is not a mesh instance")

    def session_cuda_update(self, kind: int, index: int = 0, rgb=(0.0, 0.0, 0.0)):
        """Edits the reference scene (kind 1: material `index`'s Disney base colour; kind 2:
        AreaLight `index`'s radiance; kind 3: nothing, the instances were moved by move_instance)
        and calls the adapter's RenderDevice::updateScene with that SceneUpdateKind."""
        rc = self.lib.ref_session_cuda_update(self.h, int(kind), int(index), _f3(rgb))
        if rc != 0:
            raise RuntimeError(f"adapter update failed ({rc})")

    def render_into(self, film: "RefFilm", camera, settings, first: int, count: int, threads: int = 0) -> int:
        """Renderer::renderSamples (seed 12345) adding samples [first, first+count) to a kept film
        (adaptive sampling reads it); returns the samples traced."""
        return int(self.lib.ref_render_film(self.h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()), first,
                                            count, threads, film.h))

    def render_crypto(self, camera, settings, first: int, count: int, k: int = 8, threads: int = 0):
        """CryptoFilm::pixelRanks of the object and material films after renderSamples with passes
        (seed 12345): (2, h, w, k, 2) of (id, coverage), unused entries 0."""
        out = np.zeros((2, settings.height, settings.width, k, 2), np.float32)
        self.lib.ref_render_crypto(self.h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()), first, count,
                                   threads, _f(out), k)
        return out

    def render_passes(self, camera, settings, first: int, count: int, threads: int = 0):
        """Renderer::renderSamples with RenderPassFilms (seed 12345): mean beauty, counts, the eight
        light passes (8, h, w, 3), the data passes (depth, position, object id, material id) and
        the light groups (G, h, w, 3)."""
        h, w = settings.height, settings.width
        mean = np.zeros((h, w, 3), np.float32)
        cnt = np.zeros((h, w), np.uint32)
        light = np.zeros((8, h, w, 3), np.float32)
        data = np.zeros((4, h, w, 3), np.float32)
        groups = np.zeros((16, h, w, 3), np.float32)
        n = self.lib.ref_render_passes(self.h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()), first, count,
                                       threads, _f(mean), cnt.ctypes.data_as(UP), _f(light), _f(data), _f(groups), 16)
        return mean, cnt, light, data, groups[:n]

    def render_aovs(self, camera, settings, first: int, count: int, threads: int = 0):
        """Renderer::renderSamples with AovFilms (seed 12345): mean beauty, albedo, normal, alpha
        and the counts."""
        h, w = settings.height, settings.width
        out = [np.zeros((h, w, 3), np.float32) for _ in range(4)]
        cnt = np.zeros((h, w), np.uint32)
        acnt = np.zeros((h, w), np.uint32)
        self.lib.ref_render_aovs(self.h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()), first, count,
                                 threads, _f(out[0]), cnt.ctypes.data_as(UP), _f(out[1]), _f(out[2]), _f(out[3]),
                                 acnt.ctypes.data_as(UP))
        return out[0], out[1], out[2], out[3], cnt, acnt

    def render_guided(self, camera, settings, first: int, count: int, threads: int = 0):
        """Renderer::renderSamples with SD-tree path guiding on (a fresh field, trained over the
        first 32 samples)."""
        h, w = settings.height, settings.width
        mean = np.zeros((h, w, 3), np.float32)
        cnt = np.zeros((h, w), np.uint32)
        self.lib.ref_render_guided(self.h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()), first, count,
                                   threads, _f(mean), cnt.ctypes.data_as(UP))
        return mean, cnt

    def render_rows(self, camera, settings, first: int, count: int, y0: int, y1: int, threads: int = 0):
        """tracePixel loop over rows [y0, y1) only (a bounded sample of the full-frame workload)."""
        h, w = settings.height, settings.width
        mean = np.zeros((h, w, 3), np.float32)
        cnt = np.zeros((h, w), np.uint32)
        self.lib.ref_render_rows(self.h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()), first, count, threads,
                                 y0, y1, _f(mean), cnt.ctypes.data_as(UP))
        return mean, cnt

    def trace_rays(self, origins, directions, t_max, mode: int = 0, mask: int = 0x1F, time: float = 0.0):
        """Scene::intersect (mode 0) / intersectAny (mode 2) of rays: (shape, prim, t) arrays."""
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        tm = np.ascontiguousarray(t_max, np.float32).reshape(-1)
        n = o.shape[0]
        shape = np.empty(n, np.int32)
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        self.lib.ref_trace_rays(self.h, _f(o), _f(d), _f(tm), n, int(mode), int(mask), float(time),
                                shape.ctypes.data_as(IP), prim.ctypes.data_as(IP), _f(t))
        return shape, prim, t

    def trace_primary(self, camera, settings, sample_index: int = 0):
        n = settings.width * settings.height
        shape = np.empty(n, np.int32)
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        self.lib.ref_trace_primary(self.h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()), sample_index,
                                   shape.ctypes.data_as(IP), prim.ctypes.data_as(IP), _f(t))
        return shape, prim, t

    def bsdf_probe(self, material, queries, result_type):
        n = len(queries)
        q = (type(queries[0]) * n)(*queries)
        r = (result_type * n)()
        rc = self.lib.ref_bsdf_probe(self.h, self.mat_index[id(material)], q, n, r)
        if rc != 0:
            raise RuntimeError("ref_bsdf_probe failed")
        return list(r)

    def light_pick(self, p, n, u):
        p = np.ascontiguousarray(p, np.float32)
        n = np.ascontiguousarray(n, np.float32)
        u = np.ascontiguousarray(u, np.float32)
        k = len(u)
        idx = np.empty(k, np.int32)
        pmf = np.empty(k, np.float32)
        chk = np.empty(k, np.float32)
        self.lib.ref_light_pick(self.h, _f(p), _f(n), _f(u), k, idx.ctypes.data_as(IP), _f(pmf), _f(chk))
        return idx, pmf, chk

    def env_eval(self, dirs):
        dirs = np.ascontiguousarray(dirs, np.float32)
        k = dirs.shape[0]
        rgb = np.empty((k, 3), np.float32)
        pdf = np.empty(k, np.float32)
        self.lib.ref_env_eval(self.h, _f(dirs), k, _f(rgb), _f(pdf))
        return rgb, pdf


def camera_perspective(position, target, up, vfov, aspect, camera_struct):
    """The reference PerspectiveCamera's describeGpu() written into ``camera_struct``."""
    _load().ref_camera_perspective(_f3(position), _f3(target), _f3(up), vfov, aspect, C.byref(camera_struct))
    return camera_struct


def sobol(seed: int, px, py, index, n_dims: int) -> np.ndarray:
    px = np.ascontiguousarray(px, np.int32)
    py = np.ascontiguousarray(py, np.int32)
    index = np.ascontiguousarray(index, np.int32)
    out = np.empty((len(px), n_dims, 2), np.float32)
    _load().ref_sobol(seed, px.ctypes.data_as(IP), py.ctypes.data_as(IP), index.ctypes.data_as(IP), len(px), n_dims,
                      _f(out))
    return out


def _abi():
    """The C ABI's structure layouts (include/photon_cuda.h), from the package's ctypes binding
    loaded by file path: that module declares structures only and loads no library."""
    import importlib.util
    import sys
    name = "_photon_abi_structs"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, HERE.parent / "photon-engine_b200" / "_capi.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


class DescSettings:
    """RenderSettings of a scene description (the fields the reference's renderer reads)."""

    def __init__(self, d: dict):
        self.width, self.height = int(d["width"]), int(d["height"])
        self.max_bounces = int(d.get("max_bounces", 8))
        self.rr_depth = int(d.get("rr_depth", 3))
        self.shadow_quality = int(d.get("shadow_quality", 1))
        self.filter_type = int(d.get("filter_type", 3))
        self.filter_width = float(d.get("filter_width", 1.5))
        self.seed = int(d.get("seed", 12345))

    def to_c(self):
        return _abi().pe_settings(self.width, self.height, self.max_bounces, self.rr_depth, self.shadow_quality,
                                  self.filter_type, self.filter_width, 0.0, self.seed, 0.0, 0, 0.02, 16)


class DescCamera:
    """The reference's own PerspectiveCamera of a scene description."""

    def __init__(self, d: dict, fast: bool = False):
        self.lib = _load(fast)
        p = np.array([*d["position"], *d["target"], *d["up"], d["vfov"], d["aspect"]], np.float32)
        self.h = self.lib.ref_camera_create(0, _f(p))

    def __del__(self):
        try:
            self.lib.ref_camera_destroy(self.h)
        except Exception:
            pass


def ref_scene_from_description(desc: dict, fast: bool = False) -> "RefScene":
    """The reference's Scene built from a plain scene description (photon-engine_b200/scenegen.py)
    through the reference's own Scene API, with no product code or library involved: materials
    in first-use order, then shapes and area lights in op order, then the environment."""
    lib = _load(fast)
    abi = _abi()
    rs = RefScene.__new__(RefScene)
    rs.lib = lib
    rs.h = lib.ref_scene_create()
    order = []
    for kind, o in desc["ops"]:
        if kind == "mesh" and o["material"] not in order:
            order.append(o["material"])
    index = {}
    for k in order:
        d = desc["materials"][k]
        m = abi.pe_material()
        lib.ref_material_defaults(int(d["type"]), C.byref(m))
        for key, value in d.items():
            if key != "type":
                setattr(m, key, _f3(value) if isinstance(value, (tuple, list, np.ndarray)) else value)
        index[k] = lib.ref_scene_add_material(rs.h, C.byref(m))
        if index[k] < 0:
            raise RuntimeError("reference rejected a material")
    rs.mat_index = index
    for kind, o in desc["ops"]:
        if kind == "mesh":
            pos = np.ascontiguousarray(o["positions"], np.float32)
            idx = np.ascontiguousarray(o["indices"], np.uint32)
            nrm = o.get("normals")
            uv = o.get("uvs")
            nrm = None if nrm is None else np.ascontiguousarray(nrm, np.float32)
            uv = None if uv is None else np.ascontiguousarray(uv, np.float32)
            rc = lib.ref_scene_add_mesh(rs.h, _f(pos), pos.shape[0], _f(nrm), _f(uv), idx.ctypes.data_as(UP),
                                        idx.shape[0], index[o["material"]])
        else:
            rc = lib.ref_scene_add_area_light(rs.h, _f3(o["position"]), _f3(o["u"]), _f3(o["v"]), _f3(o["radiance"]),
                                              1)
        if rc != 0:
            raise RuntimeError("reference rejected a shape")
    env = desc.get("environment")
    if env is not None:
        img = np.ascontiguousarray(env["image"], np.float32)
        lib.ref_scene_set_environment(rs.h, _f(img), img.shape[1], img.shape[0], float(env["rotation"]),
                                      float(env["intensity"]), None, 1.0, None)
    lib.ref_scene_set_background(rs.h, 0, _f3((0.18, 0.18, 0.18)))
    lib.ref_scene_build(rs.h)
    return rs


class ProjectCamera:
    """The reference's camera of a loaded project (ref_camera_create parameters)."""

    def __init__(self, kind: int, params):
        self.kind = int(kind)
        self.params = [float(x) for x in params]

    def reference_params(self):
        n = {0: 11, 1: 15, 2: 11}[self.kind]
        return self.kind, self.params[:n]

    def describe_gpu(self):
        return describe_reference_camera(self)


def load_project(path, width: int, height: int):
    """The reference's loadProject + buildRenderScene of a .photon file: (RefScene, camera,
    max bounces, filter type, filter width)."""
    lib = _load()
    kind = C.c_int32(0)
    cam = (C.c_float * 16)()
    mb, ft = C.c_int32(0), C.c_int32(0)
    fw = C.c_float(0.0)
    err = C.create_string_buffer(1024)
    h = lib.ref_load_project(str(path).encode(), float(width) / float(height), C.byref(kind), cam, C.byref(mb),
                             C.byref(ft), C.byref(fw), err, len(err))
    if not h:
        raise RuntimeError(f"reference loadProject failed: {err.value.decode(errors='replace')}")
    rs = RefScene.__new__(RefScene)
    rs.lib = lib
    rs.h = h
    return rs, ProjectCamera(kind.value, list(cam)), mb.value, ft.value, fw.value


def scene_shapes(ref: "RefScene"):
    """(kind, triangles, bounds (n, 6)) of each shape of a reference scene (kind 0 mesh, 1 sphere,
    2 area-light triangle, 3 other)."""
    n = ref.lib.ref_scene_shapes(ref.h, None, None, None, 0)
    kind = np.zeros(n, np.int32)
    tris = np.zeros(n, np.int32)
    b = np.zeros((n, 6), np.float32)
    ref.lib.ref_scene_shapes(ref.h, kind.ctypes.data_as(IP), tris.ctypes.data_as(IP), _f(b), n)
    return kind, tris, b


def render_stock(ref: "RefScene", camera: DescCamera, settings: DescSettings, first: int, count: int,
                 threads: int = 0):
    """Renderer::renderSamples (the stock CPU path, Sobol seed 12345) of samples
    [first, first+count): mean image (h, w, 3) and counts."""
    h, w = settings.height, settings.width
    mean = np.zeros((h, w, 3), np.float32)
    cnt = np.zeros((h, w), np.uint32)
    ref.lib.ref_render_camera(ref.h, camera.h, C.byref(settings.to_c()), first, count, threads, _f(mean),
                              cnt.ctypes.data_as(UP))
    return mean, cnt


def cpu_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


# ---- the C restatement (pe_oracle.c): Lambert + emissive-triangle scenes --------------------
class CamDesc(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("lower_left", C.c_float * 3), ("horizontal", C.c_float * 3),
                ("vertical", C.c_float * 3)]


def _load_restatement():
    if "restatement" in _libs:
        return _libs["restatement"]
    if not RESTATEMENT_LIB.exists():
        raise RuntimeError(f"{RESTATEMENT_LIB} missing: build it with `make -C oracle restatement`")
    lib = C.CDLL(str(RESTATEMENT_LIB))
    P = C.c_void_p
    sig = {
        "po_scene_create": (P, []),
        "po_scene_destroy": (None, [P]),
        "po_scene_add_mesh": (C.c_int32, [P, FP, C.c_uint32, UP, C.c_uint32, FP, FP]),
        "po_sobol": (C.c_int32, [C.c_uint64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, FP]),
        "po_trace_primary": (C.c_int32, [P, C.POINTER(CamDesc), C.c_int32, C.c_int32, C.c_uint64, C.c_int32, IP, FP]),
        "po_render": (C.c_int32, [P, C.POINTER(CamDesc), C.c_int32, C.c_int32, C.c_uint64, C.c_int32, C.c_int32,
                                  C.c_int32, C.c_int32, C.c_int32, C.c_int32, FP]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _libs["restatement"] = lib
    return lib


def restatement_available() -> bool:
    return RESTATEMENT_LIB.exists()


def restated_sobol(seed: int, px: int, py: int, index: int, n_dims: int) -> np.ndarray:
    out = np.empty((n_dims, 2), np.float32)
    _load_restatement().po_sobol(seed, px, py, index, n_dims, _f(out))
    return out


class Restatement:
    """The C restatement holding a product Scene made of Lambert meshes (emissive or not)."""

    def __init__(self, scene):
        self.lib = _load_restatement()
        self.h = self.lib.po_scene_create()
        self.first_tri = []
        n = 0
        for kind, obj in scene.ops:
            if kind != "mesh" or obj.material.struct.type != 0:
                raise ValueError("the restatement covers Lambert meshes only")
            m = obj.material.struct
            alb = np.array(m.base_color[:], np.float32)
            emi = np.array(m.emission[:], np.float32)
            self.lib.po_scene_add_mesh(self.h, _f(obj.positions), obj.positions.shape[0],
                                       obj.indices.ctypes.data_as(UP), obj.indices.shape[0], _f(alb), _f(emi))
            self.first_tri.append(n)
            n += obj.indices.shape[0]
        self.first_tri = np.array(self.first_tri + [n])

    def __del__(self):
        try:
            self.lib.po_scene_destroy(self.h)
        except Exception:
            pass

    @staticmethod
    def _cam(camera):
        g = camera.describe_gpu()
        c = CamDesc()
        c.position[:] = g.position[:]
        c.lower_left[:] = g.lower_left[:]
        c.horizontal[:] = g.horizontal[:]
        c.vertical[:] = g.vertical[:]
        return c

    def trace_primary(self, camera, settings, sample_index: int = 0):
        """(shape, prim, t) per pixel, shapes numbered in insertion order like the device's."""
        n = settings.width * settings.height
        tri = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        self.lib.po_trace_primary(self.h, C.byref(self._cam(camera)), settings.width, settings.height, settings.seed,
                                  sample_index, tri.ctypes.data_as(IP), _f(t))
        shape = np.where(tri >= 0, np.searchsorted(self.first_tri, tri, side="right") - 1, -1).astype(np.int32)
        prim = np.where(tri >= 0, tri - self.first_tri[np.maximum(shape, 0)], -1).astype(np.int32)
        return shape, prim, t

    def render(self, camera, settings, first: int, count: int, y0: int = 0, y1: int | None = None):
        h, w = settings.height, settings.width
        mean = np.zeros((h, w, 3), np.float32)
        self.lib.po_render(self.h, C.byref(self._cam(camera)), w, h, settings.seed, settings.max_bounces,
                           settings.rr_depth, first, count, y0, h if y1 is None else y1, _f(mean))
        return mean


def dtree_probe(dirs1, rad1, dirs2, rad2, qdirs, qu, fast: bool = False):
    """The reference's DirectionalTree after two training passes (splats, buildFrom, splats,
    buildFrom): pdf of each query direction and (direction, pdf) of each query sample."""
    lib = _load(fast)
    a = [np.ascontiguousarray(x, np.float32) for x in (dirs1, rad1, dirs2, rad2, qdirs, qu)]
    nq = len(a[4])
    pdf = np.zeros(nq, np.float32)
    smp = np.zeros((nq, 4), np.float32)
    lib.ref_dtree_probe(_f(a[0]), _f(a[1]), len(a[1]), _f(a[2]), _f(a[3]), len(a[3]), _f(a[4]), _f(a[5]), nq,
                        _f(pdf), _f(smp))
    return pdf, smp


def reference_camera(camera, lib=None):
    """The reference's own camera object equal to a product camera (caller destroys it)."""
    lib = lib or _load()
    kind, params = camera.reference_params()
    p = np.asarray(params, np.float32)
    cam = lib.ref_camera_create(int(kind), _f(p))
    end = getattr(camera, "shutter_end", None)
    if end is not None:  # Camera::setShutterEnd from the end camera's own description
        e = reference_camera(end, lib)
        lib.ref_camera_set_shutter_end(cam, e)
        lib.ref_camera_destroy(e)
    return cam


def describe_reference_camera(camera):
    """Camera::describeGpu of the reference's own camera class, as a pe_camera."""
    lib = _load()
    cam = reference_camera(camera, lib)
    out = _abi().pe_camera()
    try:
        lib.ref_camera_describe(cam, C.byref(out))
    finally:
        lib.ref_camera_destroy(cam)
    return out

