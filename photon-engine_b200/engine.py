"""Host-side mirror of the reference engine's render API over the B200 C ABI.

Names, argument meaning and error behaviour follow the reference's classes so code written
against them reads the same here:

=========================  ===============================================================
reference                  here
=========================  ===============================================================
Lambertian, DisneyMaterial, Dielectric, Mirror (src/materials/*.h)    same names
TriangleMesh (src/geometry/mesh.h:17-44)                               TriangleMesh
AreaLight (src/lights/area_light.h:18-60)                              AreaLight
EnvironmentLight (src/lights/environment_light.h:42-153)               EnvironmentLight
Scene::addShape / addLight / setEnvironment / setBackground /
  buildAccelerator (src/engine/scene.h:36-62)                          Scene
PerspectiveCamera (src/camera/perspective_camera.h:14-35)              PerspectiveCamera
RenderSettings (src/engine/render_settings.h:19-47)                    RenderSettings
Film (src/core/image/film.h:23-76)                                     Film
RenderDevice / DeviceInfo / DeviceFeatures /
  RenderTargets (src/engine/render_device.h:37-86)                     CudaDevice etc.
enumerateDevices / createDevice (render_device.cpp:80-157)             enumerate_devices / create_device
RenderSession / SessionConfig (src/engine/render_session.h:34-98)      RenderSession / SessionConfig
=========================  ===============================================================

createDevice returns None and fills the error for an unusable id, as the reference does.
There is no CPU fallback behind CudaDevice: every render goes through libphoton_cuda.so.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import enum
import math
import threading
import time
from typing import Optional

import numpy as np

from . import _capi as capi


def _lib():
    return capi.load()


# ---------------------------------------------------------------------------------------------
# materials
class Material:
    kind = -1
    _maps = ("albedo", "roughness", "metalness", "normal", "opacity")

    def __init__(self):
        self._m = capi.pe_material()
        _lib().pe_material_defaults(self.kind, C.byref(self._m))
        self.images: dict[str, np.ndarray] = {}
        self.mipmapped: set[int] = set()  # ids of images given with mipmaps
        self.linear_u8: set[int] = set()  # ids of 8-bit images stored linear (not sRGB)

    @property
    def struct(self) -> capi.pe_material:
        return self._m

    def struct_with(self, texture_index) -> capi.pe_material:
        """The material's C description with its image maps numbered by `texture_index`
        (id of the image array → index of pe_scene_add_texture)."""
        m = capi.pe_material()
        C.memmove(C.byref(m), C.byref(self._m), C.sizeof(m))
        for k, img in self.images.items():
            setattr(m, k + "_texture", texture_index[id(img)])
        return m

    def emitted(self):
        return tuple(self._m.emission)

    def set_round_edge_radius(self, r):
        """Material::setRoundEdgeRadius: shading normals blend with the neighbouring faces within
        this distance of an edge (first three vertices of a path)."""
        self._m.round_edge_radius = max(0.0, float(r))


class Lambertian(Material):
    kind = capi.PE_MAT_LAMBERT

    def __init__(self, albedo, emission=(0.0, 0.0, 0.0)):
        super().__init__()
        self._m.base_color = capi.f3(albedo)
        self._m.emission = capi.f3(emission)


class DisneyMaterial(Material):
    kind = capi.PE_MAT_DISNEY

    def _set_image(self, key, image, mipmaps, srgb=True):
        # float images are linear; uint8 images are sRGB-encoded unless srgb=False
        # (Image::createCompact8 with U8Srgb / U8Linear)
        src = np.asarray(image)
        img = np.ascontiguousarray(src, dtype=np.uint8 if src.dtype == np.uint8 else np.float32)
        if img.ndim != 3 or img.shape[2] != 3:
            raise ValueError("image maps are (height, width, 3) arrays")
        self.images[key] = img
        if img.dtype == np.uint8 and not srgb:
            self.linear_u8.add(id(img))
        if mipmaps:
            self.mipmapped.add(id(img))

    # `mipmaps`: Image::buildMipmaps on the image, so that lookups pick a level from the ray cone
    def set_albedo_image(self, image, mipmaps: bool = False, srgb: bool = True):
        """DisneyMaterial::setAlbedoImage: the base colour from an RGB image (float, or uint8
        sRGB-encoded unless srgb=False)."""
        self._set_image("albedo", image, mipmaps, srgb)

    def set_roughness_image(self, image, mipmaps: bool = False, srgb: bool = False):
        """DisneyMaterial::setRoughnessImage: roughness from the image's green channel."""
        self._set_image("roughness", image, mipmaps, srgb)

    def set_metalness_image(self, image, mipmaps: bool = False, srgb: bool = False):
        """DisneyMaterial::setMetalnessImage: metalness from the image's blue channel."""
        self._set_image("metalness", image, mipmaps, srgb)

    def set_normal_image(self, image, mipmaps: bool = False, srgb: bool = False):
        """DisneyMaterial::setNormalImage: a tangent-space normal map."""
        self._set_image("normal", image, mipmaps, srgb)

    def set_opacity_image(self, image):
        """DisneyMaterial::setOpacityImage: coverage = opacity × the image's red channel
        (cutouts for camera, bounce and shadow rays)."""
        self._set_image("opacity", image, False)

    def set_texture_mapping(self, box: bool):
        """DisneyMaterial::setTextureMapping: UV (False) or box projection (True)."""
        self._m.texture_mapping = 1 if box else 0

    def set_texture_scale(self, s: float):
        """DisneyMaterial::setTextureScale (at least 1e-4)."""
        self._m.texture_scale = max(1e-4, float(s))

    def __init__(self, base_color, metallic: float, roughness: float, specular: float = 0.5):
        super().__init__()
        self._m.base_color = capi.f3(base_color)
        self._m.metallic = metallic
        self._m.roughness = roughness
        self._m.specular = specular

    def set_clear_coat(self, v): self._m.clearcoat = v
    def set_clear_coat_roughness(self, v): self._m.clearcoat_roughness = v
    def set_ior(self, v): self._m.ior = v
    def set_specular_transmission(self, v): self._m.spec_transmission = v
    def set_coat_ior(self, v): self._m.coat_ior = v
    def set_coat_tint(self, c): self._m.coat_tint = capi.f3(c)

    def set_sheen_color(self, c):
        self._m.sheen_color = capi.f3(c)
        self._m.has_sheen_color = 1

    def set_anisotropy(self, v): self._m.anisotropy = v
    def set_sheen(self, v): self._m.sheen = v
    def set_sheen_roughness(self, v): self._m.sheen_roughness = v
    def set_diffuse_roughness(self, v): self._m.diffuse_roughness = v
    def set_diffuse_transmission(self, v): self._m.diffuse_transmission = v
    def set_subsurface(self, v): self._m.subsurface = v
    def set_subsurface_radius(self, c): self._m.subsurface_radius = capi.f3(c)
    def set_subsurface_scale(self, v): self._m.subsurface_scale = v
    def set_subsurface_anisotropy(self, v): self._m.subsurface_anisotropy = v
    def set_edge_tint(self, c): self._m.edge_tint = capi.f3(c)

    def set_thin_film(self, thickness_nm, ior):
        self._m.thin_film_thickness = thickness_nm
        self._m.thin_film_ior = ior

    def set_flakes(self, density, size, roughness, color):
        self._m.flake_density = density
        self._m.flake_size = size
        self._m.flake_roughness = roughness
        self._m.flake_color = capi.f3(color)

    def set_emission(self, c): self._m.emission = capi.f3(c)
    def set_opacity(self, v): self._m.opacity = v


class Dielectric(Material):
    kind = capi.PE_MAT_DIELECTRIC

    def __init__(self, ior: float, tint=(1.0, 1.0, 1.0), roughness: float = 0.0):
        super().__init__()
        self._m.ior = ior
        self._m.base_color = capi.f3(tint)
        self._m.glass_roughness = roughness

    def set_abbe(self, v): self._m.abbe = v

    def set_absorption(self, color, distance):
        self._m.absorb_color = capi.f3(color)
        self._m.absorb_distance = distance
        self._m.has_absorption = 1

    def set_scattering(self, density, color, anisotropy):
        self._m.scatter_density = density
        self._m.scatter_color = capi.f3(color)
        self._m.scatter_anisotropy = anisotropy
        self._m.has_scattering = 1

    def set_thin_walled(self, v: bool): self._m.thin_walled = 1 if v else 0
    def set_thin_film(self, thickness_nm): self._m.film_thickness = thickness_nm


class Mirror(Material):
    kind = capi.PE_MAT_MIRROR

    def __init__(self, reflectance):
        super().__init__()
        self._m.base_color = capi.f3(reflectance)


# ---------------------------------------------------------------------------------------------
# shapes and lights
# VisibilityMask (src/core/math/ray.h:18-25): the ray classes a shape is seen by
VIS_CAMERA, VIS_DIFFUSE, VIS_GLOSSY, VIS_TRANSMISSION, VIS_SHADOW = 1, 2, 4, 8, 16
VIS_ALL = 0x1F


class TriangleMesh:
    def __init__(self, positions, normals=None, uvs=None, indices=None, material: Material | None = None):
        self.positions = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        self.normals = None if normals is None or len(normals) == 0 else np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
        self.uvs = None if uvs is None or len(uvs) == 0 else np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1, 2)
        self.indices = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3)
        self.material = material
        self.visibility_mask = VIS_ALL

    def set_visibility_mask(self, mask: int):
        """Shape::setVisibilityMask: VIS_CAMERA | VIS_DIFFUSE | VIS_GLOSSY | VIS_TRANSMISSION | VIS_SHADOW."""
        self.visibility_mask = int(mask) & VIS_ALL

    def num_triangles(self) -> int:
        return int(self.indices.shape[0])


class Sphere:
    """Sphere (src/geometry/sphere.h): an analytic sphere with one material."""

    def __init__(self, center, radius: float, material: Material | None = None):
        self.center = tuple(map(float, center))
        self.radius = float(radius)
        self.material = material
        self.visibility_mask = VIS_ALL

    set_visibility_mask = TriangleMesh.set_visibility_mask

    def num_triangles(self) -> int:
        return 0


class MeshInstance:
    """MeshInstance (src/geometry/mesh_instance.h): a TriangleMesh placed by a local-to-world 4×4
    matrix (row-major, column vectors; translation in the last column), with the instance's own
    material (else the mesh's).  Instances of one mesh share its BVH (a BLAS) on the device; the
    top-level tree holds one primitive per instance.  `world_to_local` is the matrix's inverse as
    the caller composed it (Transform keeps both); omitted, it is computed by Mat4f::inverse's
    cofactor expansion."""

    def __init__(self, mesh: TriangleMesh, local_to_world, material: Material | None = None, world_to_local=None):
        self.mesh = mesh
        self.local_to_world = np.ascontiguousarray(local_to_world, dtype=np.float32).reshape(4, 4)
        self.world_to_local = None if world_to_local is None else \
            np.ascontiguousarray(world_to_local, dtype=np.float32).reshape(4, 4)
        self.material = material if material is not None else mesh.material
        self.visibility_mask = VIS_ALL
        self.local_to_world_end = None
        self.world_to_local_end = None

    def set_motion_transform(self, local_to_world_end, world_to_local_end=None):
        """MeshInstance::setMotionTransform: the pose at shutter close (t = 1).  Rays at time t meet
        the instance under interpolateTransform (translation and scale linear, rotation SLERP)."""
        self.local_to_world_end = np.ascontiguousarray(local_to_world_end, dtype=np.float32).reshape(4, 4)
        self.world_to_local_end = None if world_to_local_end is None else \
            np.ascontiguousarray(world_to_local_end, dtype=np.float32).reshape(4, 4)

    def has_motion(self) -> bool:
        return self.local_to_world_end is not None

    set_visibility_mask = TriangleMesh.set_visibility_mask

    def num_triangles(self) -> int:
        return 0


class AreaLight:
    def __init__(self, position, u, v, radiance):
        self.position = tuple(map(float, position))
        self.u = tuple(map(float, u))
        self.v = tuple(map(float, v))
        self.radiance = tuple(map(float, radiance))
        self.visible_to_camera = True
        self.light_group = ""

    def set_visible_to_camera(self, v: bool):
        self.visible_to_camera = bool(v)

    def set_light_group(self, name: str):
        """Light::setLightGroup (light.h:85): the render pass (LG_<name>) this light's light goes to."""
        self.light_group = str(name)


class EnvironmentLight:
    def __init__(self, image: Optional[np.ndarray], rotation: float = 0.0, intensity: float = 1.0):
        self.image = None if image is None else np.ascontiguousarray(image, dtype=np.float32)
        self.rotation = float(rotation)
        self.intensity = float(intensity)
        self.sun = None
        self.light_group = ""

    def set_light_group(self, name: str):
        """Light::setLightGroup of the environment (its pass is LG_<name>; "Env" by default)."""
        self.light_group = str(name)

    def set_sun(self, direction, cos_max, radiance):
        self.sun = (tuple(map(float, direction)), float(cos_max), tuple(map(float, radiance)))


class BackgroundMode(enum.IntEnum):
    Environment = capi.PE_BG_ENVIRONMENT
    Color = capi.PE_BG_COLOR
    Transparent = capi.PE_BG_TRANSPARENT


@dataclasses.dataclass
class Background:
    mode: BackgroundMode = BackgroundMode.Environment
    color: tuple = (0.18, 0.18, 0.18)


class Scene:
    """Immutable-after-build render scene.  ``ops`` records the add calls in order so the same
    content can be replayed into another implementation (the parity tests do this)."""

    def __init__(self):
        self.ops: list = []
        self.environment: Optional[EnvironmentLight] = None
        self.background = Background()
        self._handle = None
        self._materials: list[Material] = []
        self._mat_index: dict[int, int] = {}
        self.info: Optional[capi.pe_scene_info] = None
        self.shadow_catcher: Optional[int] = None
        self.shape_tags: dict[int, int] = {}
        self.light_links: dict[int, tuple] = {}
        self.light_groups: dict[int, str] = {}
        self._tex_index: dict = {}
        self.shape_names: dict[int, str] = {}
        self.material_names: dict[int, tuple] = {}

    def __del__(self):
        try:
            if self._handle:
                _lib().pe_scene_destroy(self._handle)
        except Exception:
            pass

    def add_shape(self, shape):
        """Scene::addShape of a TriangleMesh or a Sphere."""
        if shape.material is None:
            raise ValueError(f"{type(shape).__name__} needs a material")
        kind = "sphere" if isinstance(shape, Sphere) else ("instance" if isinstance(shape, MeshInstance) else "mesh")
        self.ops.append((kind, shape))

    def add_light(self, light: AreaLight):
        self.ops.append(("area", light))

    def set_environment(self, env: Optional[EnvironmentLight]):
        self.environment = env

    def shape_count(self) -> int:
        """Shapes added so far: one per mesh, two per area light (its two triangles)."""
        return sum(2 if kind == "area" else 1 for kind, _ in self.ops)

    def tag_shape(self, shape: int, node_uid: int):
        """Scene::tagShape: the scene-node uid that light links name this shape by."""
        self.shape_tags[int(shape)] = int(node_uid)

    def set_light_link(self, light: int, mode: int = 0, uids=(), shadow_mode: int = 0, shadow_uids=()):
        """Light::setLightLink of explicit light `light` (one per area light, one per triangle of an
        emissive mesh, in the order they were added): mode / shadow_mode 0 all, 1 include the
        listed node uids, 2 exclude them."""
        self.light_links[int(light)] = (int(mode), [int(u) for u in uids], int(shadow_mode),
                                        [int(u) for u in shadow_uids])

    def set_shape_name(self, shape: int, name: str):
        """Scene::setShapeName: the name the shape's Cryptomatte id hashes."""
        self.shape_names[int(shape)] = str(name)

    def set_material_name(self, material, name: str):
        """Scene::setMaterialName: the name the material's Cryptomatte id hashes."""
        self.material_names[id(material)] = (material, str(name))

    def set_light_group(self, light: int, name: str):
        """Light::setLightGroup of light `light` (numbered as set_light_link numbers them); an
        AreaLight's own set_light_group does the same for it."""
        self.light_groups[int(light)] = str(name)

    def light_group_names(self) -> list[str]:
        """Scene::lightGroupNames of the built scene (scene.cpp:144-174)."""
        lib = _lib()
        n = lib.pe_scene_light_groups(self.handle, None, 0)
        if n < 0:
            capi.check(n)
        buf = C.create_string_buffer(16 * 256)
        lib.pe_scene_light_groups(self.handle, buf, len(buf))
        return [x.decode() for x in buf.raw.split(b"\0")[:n]]

    def set_shadow_catcher(self, shape: Optional[int]):
        """Scene::setShadowCatcher: camera rays see this shape (an index as counted by
        shape_count at the time it was added) as the background darkened by its shadows."""
        self.shadow_catcher = shape

    def set_background(self, bg: Background):
        self.background = bg

    def materials(self) -> list[Material]:
        out, seen = [], set()
        for kind, obj in self.ops:
            if kind in ("mesh", "sphere", "instance") and id(obj.material) not in seen:
                seen.add(id(obj.material))
                out.append(obj.material)
        return out

    def textures(self) -> list:
        """The image maps of the scene's materials, each once, in material order."""
        out, seen = [], set()
        for m in self.materials():
            for k in Material._maps:
                img = getattr(m, "images", {}).get(k)
                if img is not None and id(img) not in seen:
                    seen.add(id(img))
                    out.append(img)
        return out

    def sync_materials(self) -> bool:
        """Sends every material's current parameters to the built scene without rebuilding it
        (pe_scene_set_material); False when some change needs a rebuild (type, emission, media,
        shadow or walk switches, a new image)."""
        if not self._handle:
            return False
        lib = _lib()
        for m in self.materials():
            idx = self._mat_index.get(id(m))
            if idx is None or any(id(img) not in self._tex_index for img in getattr(m, "images", {}).values()):
                return False
            if lib.pe_scene_set_material(self._handle, idx, C.byref(m.struct_with(self._tex_index))) != capi.PE_OK:
                return False
        return True

    def sync_lights(self) -> bool:
        """Sends every AreaLight's current radiance to the built scene without rebuilding its BVH
        (pe_scene_set_area_light_radiance); False when that is not possible."""
        if not self._handle:
            return False
        lib, li = _lib(), 0
        for kind, obj in self.ops:
            if kind == "sphere":
                continue
            if kind in ("mesh", "instance"):
                m = obj.material.struct
                if m.type in (capi.PE_MAT_LAMBERT, capi.PE_MAT_DISNEY) and any(m.emission):
                    li += (obj.mesh if kind == "instance" else obj).indices.shape[0]
            else:
                if lib.pe_scene_set_area_light_radiance(self._handle, li, capi.f3(obj.radiance)) != capi.PE_OK:
                    return False
                li += 1
        return True

    def sync_transforms(self) -> bool:
        """Sends every MeshInstance's current matrices to the built scene
        (pe_scene_set_instance_transform); False when that is not possible (an emissive instance)."""
        if not self._handle:
            return False
        lib = _lib()
        shape = 0
        for kind, obj in self.ops:
            if kind == "instance":
                if lib.pe_scene_set_instance_transform(self._handle, shape, capi.fptr(obj.local_to_world),
                                                       capi.fptr(obj.world_to_local)) != capi.PE_OK:
                    return False
            shape += 2 if kind == "area" else 1
        return True

    def texture_has_mipmaps(self, img) -> bool:
        return any(id(img) in getattr(m, "mipmapped", ()) for m in self.materials())

    def build_accelerator(self):
        lib = _lib()
        if self._handle:
            lib.pe_scene_destroy(self._handle)
        h = lib.pe_scene_create()
        if not h:
            raise MemoryError("pe_scene_create failed")
        self._handle = h
        tex_index = {}
        for img in self.textures():
            if img.dtype == np.uint8:
                srgb = not any(id(img) in getattr(m, "linear_u8", ()) for m in self.materials())
                t = lib.pe_scene_add_texture_u8(h, img.ctypes.data_as(C.POINTER(C.c_uint8)), img.shape[1], img.shape[0],
                                                1 if srgb else 0)
            else:
                t = lib.pe_scene_add_texture(h, capi.fptr(img), img.shape[1], img.shape[0])
            if t < 0:
                capi.check(t)
            if self.texture_has_mipmaps(img):
                capi.check(lib.pe_scene_build_texture_mipmaps(h, t))
            tex_index[id(img)] = t
        self._tex_index = tex_index
        mat_index = {}
        blas_index = {}
        for m in self.materials():
            idx = lib.pe_scene_add_material(h, C.byref(m.struct_with(tex_index)))
            if idx < 0:
                capi.check(capi.PE_ERR_INVALID)
            mat_index[id(m)] = idx
        self._mat_index = mat_index
        shape_count = 0
        for kind, obj in self.ops:
            if kind == "mesh":
                capi.check(lib.pe_scene_add_mesh(h, capi.fptr(obj.positions), obj.positions.shape[0],
                                                 capi.fptr(obj.normals), capi.fptr(obj.uvs), capi.uptr(obj.indices),
                                                 obj.indices.shape[0], mat_index[id(obj.material)]))
            elif kind == "sphere":
                capi.check(lib.pe_scene_add_sphere(h, capi.f3(obj.center), obj.radius, mat_index[id(obj.material)]))
            elif kind == "instance":
                mesh = obj.mesh
                b = blas_index.get(id(mesh))
                if b is None:
                    b = lib.pe_scene_add_blas(h, capi.fptr(mesh.positions), mesh.positions.shape[0],
                                              capi.fptr(mesh.normals), capi.fptr(mesh.uvs), capi.uptr(mesh.indices),
                                              mesh.indices.shape[0])
                    if b < 0:
                        capi.check(-b)
                    blas_index[id(mesh)] = b
                capi.check(lib.pe_scene_add_instance(h, b, capi.fptr(obj.local_to_world), capi.fptr(obj.world_to_local),
                                                     mat_index[id(obj.material)]))
                if obj.has_motion():
                    capi.check(lib.pe_scene_set_instance_motion(h, shape_count, capi.fptr(obj.local_to_world_end),
                                                                capi.fptr(obj.world_to_local_end)))
            else:
                capi.check(lib.pe_scene_add_area_light(h, capi.f3(obj.position), capi.f3(obj.u), capi.f3(obj.v),
                                                       capi.f3(obj.radiance), 1 if obj.visible_to_camera else 0))
            shape_count += 2 if kind == "area" else 1
        if self.shadow_catcher is not None:
            capi.check(lib.pe_scene_set_shadow_catcher(h, int(self.shadow_catcher)))
        for shape, uid in self.shape_tags.items():
            capi.check(lib.pe_scene_tag_shape(h, shape, uid))
        for shape, name in self.shape_names.items():
            capi.check(lib.pe_scene_set_shape_name(h, shape, name.encode()))
        shape = 0
        for kind, obj in self.ops:
            if kind != "area" and obj.visibility_mask != VIS_ALL:
                capi.check(lib.pe_scene_set_shape_visibility(h, shape, obj.visibility_mask))
            shape += 2 if kind == "area" else 1
        for mat, name in self.material_names.values():
            if id(mat) in mat_index:
                capi.check(lib.pe_scene_set_material_name(h, mat_index[id(mat)], name.encode()))
        groups, li = {}, 0
        for kind, obj in self.ops:
            if kind == "sphere":
                continue
            if kind in ("mesh", "instance"):
                m = obj.material.struct
                if m.type in (capi.PE_MAT_LAMBERT, capi.PE_MAT_DISNEY) and any(m.emission):
                    li += (obj.mesh if kind == "instance" else obj).indices.shape[0]
            else:
                if obj.light_group:
                    groups[li] = obj.light_group
                li += 1
        groups.update(self.light_groups)
        for light, name in groups.items():
            capi.check(lib.pe_scene_set_light_group(h, light, name.encode()))
        for light, (mode, uids, smode, suids) in self.light_links.items():
            a = (C.c_uint64 * max(1, len(uids)))(*uids)
            b = (C.c_uint64 * max(1, len(suids)))(*suids)
            capi.check(lib.pe_scene_set_light_link(h, light, mode, a, len(uids), smode, b, len(suids)))
        env = self.environment
        if env is not None:
            img = env.image
            if img is not None:
                capi.check(lib.pe_scene_set_environment(h, capi.fptr(img), img.shape[1], img.shape[0], env.rotation,
                                                        env.intensity))
            else:
                capi.check(lib.pe_scene_set_environment(h, None, 0, 0, env.rotation, env.intensity))
            if env.sun is not None:
                d, cm, r = env.sun
                capi.check(lib.pe_scene_set_sun(h, capi.f3(d), cm, capi.f3(r)))
            if env.light_group:
                capi.check(lib.pe_scene_set_light_group(h, -1, env.light_group.encode()))
        capi.check(lib.pe_scene_set_background(h, int(self.background.mode), capi.f3(self.background.color)))
        capi.check(lib.pe_scene_build(h))
        info = capi.pe_scene_info()
        capi.check(lib.pe_scene_get_info(h, C.byref(info)))
        self.info = info
        return self

    @property
    def handle(self):
        if not self._handle:
            raise RuntimeError("Scene.build_accelerator() has not been called")
        return self._handle


# ---------------------------------------------------------------------------------------------
class PerspectiveCamera:
    def __init__(self, position, target, up, vfov_degrees: float, aspect: float):
        self.position, self.target, self.up = position, target, up
        self.vfov, self.aspect = float(vfov_degrees), float(aspect)
        self._desc = capi.pe_camera()
        _lib().pe_camera_perspective(capi.f3(position), capi.f3(target), capi.f3(up), self.vfov, self.aspect,
                                     C.byref(self._desc))

    def describe_gpu(self) -> capi.pe_camera:
        return self._desc

    def set_shutter_end(self, end: "PerspectiveCamera"):
        """Camera::setShutterEnd: `end`'s pose at shutter close (t = 1).  With motion blur a ray at
        time t > 0 mixes the two descriptions linearly (a round lens of the mixed radius)."""
        e = end.describe_gpu()
        d = self._desc
        d.has_shutter_end = 1
        for f in ("position", "lower_left", "horizontal", "vertical", "u", "v", "forward"):
            setattr(d, "end_" + f, capi.f3(tuple(getattr(e, f))))
        d.end_lens_radius = e.lens_radius
        self.shutter_end = end

    def has_shutter_end(self) -> bool:
        return bool(self._desc.has_shutter_end)

    def reference_params(self):
        """(kind, parameters) of the same camera in the reference's own classes (test oracle)."""
        return 0, [*self.position, *self.target, *self.up, self.vfov, self.aspect]


class ThinLensCamera(PerspectiveCamera):
    """ThinLensCamera: depth of field (aperture radius, focus distance), optionally a polygonal
    aperture of `blades` sides rotated by `rotation_degrees` (setApertureShape)."""

    def __init__(self, position, target, up, vfov_degrees: float, aspect: float, aperture_radius: float,
                 focus_distance: float, blades: int = 0, rotation_degrees: float = 0.0):
        self.position, self.target, self.up = position, target, up
        self.vfov, self.aspect = float(vfov_degrees), float(aspect)
        self.aperture, self.focus = float(aperture_radius), float(focus_distance)
        self.blades, self.rotation = int(blades), float(rotation_degrees)
        self._desc = capi.pe_camera()
        _lib().pe_camera_thin_lens(capi.f3(position), capi.f3(target), capi.f3(up), self.vfov, self.aspect,
                                   self.aperture, self.focus, self.blades, self.rotation, C.byref(self._desc))

    def reference_params(self):
        return 1, [*self.position, *self.target, *self.up, self.vfov, self.aspect, self.aperture, self.focus,
                   float(self.blades), self.rotation]


class OrthographicCamera(PerspectiveCamera):
    """OrthographicCamera: parallel rays over a `vertical_extent`-high image plane."""

    def __init__(self, position, target, up, vertical_extent: float, aspect: float):
        self.position, self.target, self.up = position, target, up
        self.extent, self.aspect = float(vertical_extent), float(aspect)
        self._desc = capi.pe_camera()
        _lib().pe_camera_orthographic(capi.f3(position), capi.f3(target), capi.f3(up), self.extent, self.aspect,
                                      C.byref(self._desc))

    def reference_params(self):
        return 2, [*self.position, *self.target, *self.up, self.extent, self.aspect]


class PixelFilterType(enum.IntEnum):
    Box = capi.PE_FILTER_BOX
    Triangle = capi.PE_FILTER_TRIANGLE
    Gaussian = capi.PE_FILTER_GAUSSIAN
    BlackmanHarris = capi.PE_FILTER_BLACKMAN_HARRIS


@dataclasses.dataclass
class RenderSettings:
    width: int = 512
    height: int = 512
    samples_per_pixel: int = 64
    max_bounces: int = 8
    tile_size: int = 32
    num_threads: int = 0
    adaptive_sampling: bool = False
    clamp_indirect: float = 0.0
    shadow_quality: int = 1
    filter_type: PixelFilterType = PixelFilterType.BlackmanHarris
    filter_width: float = 1.5
    seed: int = 12345            # Renderer::renderSamples uses a fixed Sobol seed of 12345
    rr_depth: int = 3            # PathTracer(maxBounces, 3, ...) in renderSamples
    path_guiding: bool = False
    ao_strength: float = 0.0     # RenderSettings::aoStrength: contact AO at camera hits
    noise_threshold: float = 0.02    # adaptive: relative standard error target (render_settings.h:31)
    min_adaptive_samples: int = 16   # adaptive: samples before any decision (render_settings.h:32)
    motion_blur: bool = False        # RenderSettings::motionBlur: a shutter time per camera sample

    def to_c(self) -> capi.pe_settings:
        return capi.pe_settings(self.width, self.height, self.max_bounces, self.rr_depth, self.shadow_quality,
                                int(self.filter_type), self.filter_width, self.clamp_indirect, self.seed,
                                float(self.ao_strength), 1 if self.adaptive_sampling else 0,
                                float(self.noise_threshold), int(self.min_adaptive_samples),
                                1 if self.motion_blur else 0)


class Film:
    """Per-pixel radiance sum, sample count and luminance² sum (src/core/image/film.h:23-76)."""

    def __init__(self, width: int = 0, height: int = 0):
        self.resize(width, height)

    def resize(self, width: int, height: int):
        self.width, self.height = max(0, width), max(0, height)
        self.sum = np.zeros((self.height, self.width, 3), np.float32)
        self.count = np.zeros((self.height, self.width), np.uint32)
        self.sum_sq = np.zeros((self.height, self.width), np.float32)
        self.rejected = 0

    def clear(self):
        self.resize(self.width, self.height)

    def resolve(self) -> np.ndarray:
        inv = np.zeros_like(self.sum_sq)
        nz = self.count > 0
        inv[nz] = 1.0 / self.count[nz].astype(np.float32)
        return self.sum * inv[..., None]

    def relative_error(self) -> np.ndarray:
        n = self.count.astype(np.float32)
        s = self.sum
        mean = (0.212671 * s[..., 0] + 0.715160 * s[..., 1] + 0.072169 * s[..., 2]) / np.maximum(n, 1)
        mean_sq = self.sum_sq / np.maximum(n, 1)
        var = np.maximum(0.0, mean_sq - mean * mean) * n / np.maximum(n - 1, 1)
        err = np.sqrt(var / np.maximum(n, 1)) / (np.maximum(mean, 0.0) + 0.01)
        return np.where(n < 2, np.float32(1e30), err)

    def merge(self, other: "Film"):
        self.sum += other.sum
        self.count += other.count
        self.sum_sq += other.sum_sq
        self.rejected += other.rejected


class AovFilms:
    """AovFilms (renderer.h:42-53): the first visible surface's albedo, its normal and coverage."""

    def __init__(self, width: int = 0, height: int = 0):
        self.albedo = Film(width, height)
        self.normal = Film(width, height)
        self.alpha = Film(width, height)

    def resize(self, width: int, height: int):
        for f in (self.albedo, self.normal, self.alpha):
            f.resize(width, height)


class LightPass(enum.IntEnum):
    """LightPass (path_tracer.h:21-24); the films' channel names are lightPassName's."""
    DiffuseDirect = 0
    DiffuseIndirect = 1
    GlossyDirect = 2
    GlossyIndirect = 3
    TransmissionDirect = 4
    TransmissionIndirect = 5
    Emission = 6
    Background = 7


class CryptoFilm:
    """CryptoFilm (cryptomatte.h): per pixel the samples taken and the count of each Cryptomatte
    id (a float hash of an object or material name) among them."""

    def __init__(self, width: int, height: int):
        self.width, self.height = width, height
        self.total = np.zeros((height, width), np.uint32)
        self.counts: dict = {}   # (y, x) → {id: count}

    def add_samples(self, ids: np.ndarray, taken: np.ndarray):
        """CryptoFilm::addSample for each sample: ids (n, h, w), taken (n, h, w) bool."""
        self.total += taken.sum(axis=0).astype(np.uint32)
        n, h, w = ids.shape
        flat = ids.reshape(n, -1)
        hit = (flat != 0.0) & taken.reshape(n, -1)
        for p in np.nonzero(hit.any(axis=0))[0]:
            vals, cnt = np.unique(flat[hit[:, p], p], return_counts=True)
            d = self.counts.setdefault((int(p) // w, int(p) % w), {})
            for v, c in zip(vals.tolist(), cnt.tolist()):
                d[v] = d.get(v, 0) + int(c)

    def pixel_ranks(self, x: int, y: int):
        """CryptoFilm::pixelRanks: (id, coverage) by falling coverage."""
        d = self.counts.get((y, x), {})
        t = int(self.total[y, x])
        if t == 0:
            return []
        return sorted(((i, c / t) for i, c in d.items()), key=lambda e: -e[1])


class RenderPassFilms:
    """RenderPassFilms (renderer.h:59-98): the eight light passes (their sum is the beauty film),
    the data passes of the first hit (depth, position, object and material id colours) and one
    film per light group, as (name, Film) pairs in Scene::lightGroupNames order."""

    def __init__(self, width: int = 0, height: int = 0):
        self.light = [Film(width, height) for _ in range(len(LightPass))]
        self.depth = Film(width, height)
        self.position = Film(width, height)
        self.object_id = Film(width, height)
        self.material_id = Film(width, height)
        self.light_groups: list[tuple[str, Film]] = []
        self.crypto_object: Optional[CryptoFilm] = None    # enable_cryptomatte
        self.crypto_material: Optional[CryptoFilm] = None

    def enable_cryptomatte(self):
        """CryptoObject and CryptoMaterial films (the reference fills them when they are sized)."""
        w, h = self.depth.width, self.depth.height
        self.crypto_object, self.crypto_material = CryptoFilm(w, h), CryptoFilm(w, h)

    def init_light_groups(self, width: int, height: int, names):
        self.light_groups = [(n, Film(width, height)) for n in names]

    def resize(self, width: int, height: int):
        for f in (*self.light, self.depth, self.position, self.object_id, self.material_id):
            f.resize(width, height)
        for _, f in self.light_groups:
            f.resize(width, height)

    def to_c(self) -> capi.pe_pass_films:
        def arr(f: Film):
            return capi.pe_film_arrays(capi.fptr(f.sum), capi.uptr(f.count), capi.fptr(f.sum_sq))
        out = capi.pe_pass_films()
        for k, f in enumerate(self.light):
            out.light[k] = arr(f)
        out.depth, out.position = arr(self.depth), arr(self.position)
        out.object_id, out.material_id = arr(self.object_id), arr(self.material_id)
        out.n_groups = len(self.light_groups)
        for g, (_, f) in enumerate(self.light_groups[:capi.PE_MAX_LIGHT_GROUPS]):
            out.groups[g] = arr(f)
        return out


@dataclasses.dataclass
class RenderTargets:
    beauty: Optional[Film] = None
    aovs: object = None
    passes: object = None


@dataclasses.dataclass
class SampleBatchResult:
    completed: bool = True
    samples_traced: int = 0


@dataclasses.dataclass
class DeviceFeatures:
    aovs: bool = True
    light_passes: bool = True
    adaptive_sampling: bool = True


class DeviceKind(enum.Enum):
    Cpu = "cpu"
    Cuda = "cuda"


@dataclasses.dataclass
class DeviceInfo:
    id: str = ""
    kind: DeviceKind = DeviceKind.Cuda
    name: str = ""
    threads: int = 0
    memory_bytes: int = 0
    compute_major: int = 0
    compute_minor: int = 0
    hardware_ray_tracing: bool = False
    usable: bool = False
    note: str = ""


class SceneUpdateKind(enum.IntEnum):
    Full = 0
    Materials = 1
    Lights = 2
    Transforms = 3


class CudaDevice:
    """RenderDevice for one B200 (``cuda:N``).  Device handles are independent; one handle is
    driven from one thread at a time (the reference's session contract)."""

    def __init__(self, ordinal: int = 0):
        lib = _lib()
        err = C.create_string_buffer(512)
        h = lib.pe_device_create(ordinal, err, len(err))
        if not h:
            raise capi.PhotonError(capi.PE_ERR_CUDA, err.value.decode())
        self._h = h
        self._scene: Optional[Scene] = None
        di = capi.pe_device_info()
        capi.check(lib.pe_device_info_get(h, C.byref(di)))
        self._info = DeviceInfo(id=f"cuda:{ordinal}", kind=DeviceKind.Cuda, name=di.name.decode(),
                                memory_bytes=di.memory_bytes, compute_major=di.compute_major,
                                compute_minor=di.compute_minor, usable=True,
                                note=f"sm_{di.compute_major}{di.compute_minor}, {di.sm_count} SMs, wavefront path tracer")
        self.pci_bus_id = di.pci_bus_id.decode()
        self.sm_count = di.sm_count
        self._lock = threading.Lock()

    def close(self):
        if getattr(self, "_h", None):
            _lib().pe_device_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self) -> DeviceInfo:
        return self._info

    def features(self) -> DeviceFeatures:
        return DeviceFeatures()

    def set_scene(self, scene: Scene):
        if scene.info is None:
            scene.build_accelerator()
        capi.check(_lib().pe_device_set_scene(self._h, scene.handle))
        self._scene = scene

    def update_scene(self, scene: Scene, kind: SceneUpdateKind = SceneUpdateKind.Full) -> bool:
        """RenderDevice::updateScene.  Materials, Lights and Transforms (MeshInstance matrices: the
        top-level tree is refitted, no BLAS rebuilt) go to the device without a rebuild when the
        change allows it (returns True); otherwise, and for Full, the scene is rebuilt and set
        again (returns False)."""
        if kind == SceneUpdateKind.Materials and self._scene is scene and scene.sync_materials():
            if _lib().pe_device_update_materials(self._h, scene.handle) == capi.PE_OK:
                return True
        if kind == SceneUpdateKind.Lights and self._scene is scene and scene.sync_lights():
            if _lib().pe_device_update_lights(self._h, scene.handle) == capi.PE_OK:
                return True
        if kind == SceneUpdateKind.Transforms and self._scene is scene and scene.sync_transforms():
            if _lib().pe_device_update_transforms(self._h, scene.handle) == capi.PE_OK:
                return True
        scene.build_accelerator()
        self.set_scene(scene)
        return False

    def has_scene(self) -> bool:
        return bool(_lib().pe_device_has_scene(self._h))

    def render(self, camera: PerspectiveCamera, settings: RenderSettings, targets: RenderTargets, first_sample: int,
               count: int, cancel=None) -> SampleBatchResult:
        film = targets.beauty
        if film is None:
            raise ValueError("RenderTargets.beauty is required")
        st = settings.to_c()
        st.width, st.height = film.width, film.height
        flag = None
        if cancel is not None:
            flag = cancel if isinstance(cancel, C.c_int32) else C.c_int32(1 if cancel else 0)
        traced = C.c_uint64(0)
        aovs = targets.aovs
        passes = targets.passes
        with self._lock:
            self._sync_guiding(settings)
            if aovs is not None and (aovs.albedo.width != film.width or aovs.albedo.height != film.height):
                aovs.resize(film.width, film.height)
            if passes is not None:
                # renderSamples sizes the passes from the film and re-forms the light groups when
                # they do not match the scene's (renderer.cpp:401-406)
                if passes.depth.width != film.width or passes.depth.height != film.height:
                    passes.resize(film.width, film.height)
                names = self._scene.light_group_names() if self._scene is not None else []
                if [n for n, _ in passes.light_groups] != names or any(
                        f.width != film.width or f.height != film.height for _, f in passes.light_groups):
                    passes.init_light_groups(film.width, film.height, names)
                pout = passes.to_c()
                crypto = None
                if passes.crypto_object is not None:
                    crypto = (np.zeros((count, film.height, film.width), np.float32),
                              np.zeros((count, film.height, film.width), np.float32))
                    pout.crypto_object, pout.crypto_material = capi.fptr(crypto[0]), capi.fptr(crypto[1])
                    counts_before = film.count.copy()
                aout = None
                if aovs is not None:
                    aout = capi.pe_aov_films(capi.fptr(aovs.albedo.sum), capi.uptr(aovs.albedo.count),
                                             capi.fptr(aovs.albedo.sum_sq), capi.fptr(aovs.normal.sum),
                                             capi.uptr(aovs.normal.count), capi.fptr(aovs.alpha.sum),
                                             capi.uptr(aovs.alpha.count), capi.fptr(aovs.alpha.sum_sq))
                rc = _lib().pe_device_render_passes(self._h, C.byref(camera.describe_gpu()), C.byref(st), first_sample,
                                                    count, C.byref(flag) if flag is not None else None,
                                                    capi.fptr(film.sum), capi.uptr(film.count), capi.fptr(film.sum_sq),
                                                    C.byref(aout) if aout is not None else None, C.byref(pout),
                                                    C.byref(traced))
                if crypto is not None and rc == capi.PE_OK:
                    # every pixel took every sample unless adaptive sampling stopped it
                    taken = np.arange(count)[:, None, None] < (film.count - counts_before)[None]
                    passes.crypto_object.add_samples(crypto[0], taken)
                    passes.crypto_material.add_samples(crypto[1], taken)
            elif aovs is not None:
                out = capi.pe_aov_films(capi.fptr(aovs.albedo.sum), capi.uptr(aovs.albedo.count),
                                        capi.fptr(aovs.albedo.sum_sq), capi.fptr(aovs.normal.sum),
                                        capi.uptr(aovs.normal.count), capi.fptr(aovs.alpha.sum),
                                        capi.uptr(aovs.alpha.count), capi.fptr(aovs.alpha.sum_sq))
                rc = _lib().pe_device_render_aovs(self._h, C.byref(camera.describe_gpu()), C.byref(st), first_sample,
                                                  count, C.byref(flag) if flag is not None else None,
                                                  capi.fptr(film.sum), capi.uptr(film.count), capi.fptr(film.sum_sq),
                                                  C.byref(out), C.byref(traced))
            else:
                rc = _lib().pe_device_render(self._h, C.byref(camera.describe_gpu()), C.byref(st), first_sample,
                                             count, C.byref(flag) if flag is not None else None, capi.fptr(film.sum),
                                             capi.uptr(film.count), capi.fptr(film.sum_sq), C.byref(traced))
        if rc == capi.PE_ERR_CANCELLED:
            return SampleBatchResult(False, traced.value)
        capi.check(rc)
        film.rejected += int(self.last_stats().rejected)
        return SampleBatchResult(True, traced.value)

    def render_region(self, camera: PerspectiveCamera, settings: RenderSettings, film: Film, region, first_sample: int,
                      count: int) -> SampleBatchResult:
        """Adds samples [first_sample, first_sample+count) to the pixels of region = (x0, y0, w, h)
        of a whole-frame film, each exactly as render() would (pe_device_render_region)."""
        self._sync_guiding(settings)
        if film.width != settings.width or film.height != settings.height:
            film.resize(settings.width, settings.height)
        x0, y0, w, h = (int(v) for v in region)
        traced = C.c_uint64(0)
        capi.check(_lib().pe_device_render_region(self._h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()),
                                                  x0, y0, w, h, first_sample, count, None, capi.fptr(film.sum),
                                                  capi.uptr(film.count), capi.fptr(film.sum_sq), C.byref(traced)))
        film.rejected += int(self.last_stats().rejected)
        return SampleBatchResult(True, traced.value)

    def _sync_guiding(self, settings: RenderSettings):
        # RenderSettings::pathGuiding (renderer.cpp:413-429): SD-tree guiding on while it is set;
        # turning it off drops the field
        mode = getattr(self, "_guide_mode", 0)
        if settings.path_guiding and mode != 2:
            self.set_guiding(2)
        elif not settings.path_guiding and mode == 2:
            self.set_guiding(0)

    def set_guiding(self, mode: int, warmup_steps: int = 0, lr: float = 0.0):
        """0 off, 1 the learned directional proposal, 2 SD-tree guiding (pe_device_set_guiding)."""
        capi.check(_lib().pe_device_set_guiding(self._h, int(mode), int(warmup_steps), float(lr)))
        self._guide_mode = int(mode)

    def sdtree_info(self) -> capi.pe_sdtree_info:
        out = capi.pe_sdtree_info()
        capi.check(_lib().pe_device_sdtree_info(self._h, C.byref(out)))
        return out

    # resident-film path (no host film traffic per batch)
    def render_resident(self, camera: PerspectiveCamera, settings: RenderSettings, first_sample: int, count: int):
        self._sync_guiding(settings)
        st = settings.to_c()
        capi.check(_lib().pe_device_render_resident(self._h, C.byref(camera.describe_gpu()), C.byref(st),
                                                    first_sample, count, None))

    def render_tile_noalloc(self, camera: PerspectiveCamera, settings: RenderSettings, x0: int, y0: int, w: int, h: int,
                            first_sample: int, count: int, sum_ptr: int, count_ptr: int, sum_sq_ptr: int):
        """Adds samples of one film rectangle into caller-owned device buffers without allocating
        device memory (for hosts that cannot allocate while they render; see
        pe_device_render_tile_noalloc in include/photon_cuda.h).  At most 32768 pixels per call."""
        capi.check(_lib().pe_device_render_tile_noalloc(self._h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()),
                                                        x0, y0, w, h, first_sample, count, sum_ptr, count_ptr, sum_sq_ptr))

    def film_clear(self):
        capi.check(_lib().pe_device_film_clear(self._h))

    def film_read(self, width: int, height: int) -> Film:
        f = Film(width, height)
        capi.check(_lib().pe_device_film_read(self._h, capi.fptr(f.sum), capi.uptr(f.count), capi.fptr(f.sum_sq)))
        return f

    def synchronize(self):
        capi.check(_lib().pe_device_synchronize(self._h))

    def last_stats(self) -> capi.pe_render_stats:
        s = capi.pe_render_stats()
        capi.check(_lib().pe_device_last_stats(self._h, C.byref(s)))
        return s

    def timer_begin(self):
        capi.check(_lib().pe_device_timer_begin(self._h))

    def timer_end(self) -> float:
        ms = C.c_float(0.0)
        capi.check(_lib().pe_device_timer_end(self._h, C.byref(ms)))
        return float(ms.value)

    def set_counting(self, on: bool):
        capi.check(_lib().pe_device_set_counting(self._h, 1 if on else 0))

    def set_tail_paths(self, paths: int):
        """Live paths at or below which a wave finishes in the per-thread tail kernel
        (-1 = one resident grid, 0 = never); the film does not depend on it."""
        capi.check(_lib().pe_device_set_tail_paths(self._h, int(paths)))

    @property
    def tail_paths(self) -> int:
        return int(_lib().pe_device_tail_paths(self._h))

    def autotune(self, camera: PerspectiveCamera, settings: RenderSettings, probe_spp: int = 4) -> int:
        """Picks the tail threshold that renders this view fastest (films are unaffected)."""
        chosen = C.c_int64(0)
        capi.check(_lib().pe_device_autotune(self._h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()),
                                             int(probe_spp), C.byref(chosen)))
        return int(chosen.value)

    def tuning(self) -> dict:
        """The device's tuning knobs (pe_tuning): tail_paths, closest_traversal, shade_budget, any_traversal,
        wave_slots."""
        t = capi.pe_tuning()
        capi.check(_lib().pe_device_get_tuning(self._h, C.byref(t)))
        return {"tail_paths": int(t.tail_paths), "closest_traversal": int(t.closest_traversal),
                "shade_budget": int(t.shade_budget), "any_traversal": int(t.any_traversal),
                "wave_slots": int(t.wave_slots)}

    def set_tuning(self, tail_paths: int = -1, closest_traversal: int = 6, shade_budget: int = 1, any_traversal: int = 2,
                   wave_slots: int = 1 << 23):
        capi.check(_lib().pe_device_set_tuning(self._h, C.byref(capi.pe_tuning(tail_paths, closest_traversal,
                                                                                shade_budget, any_traversal,
                                                                                wave_slots))))

    def autotune_log(self) -> str:
        """The last autotune's probe times ("knob=value time ms" per line)."""
        n = _lib().pe_device_autotune_log(self._h, None, 0)
        buf = C.create_string_buffer(max(1, n + 1))
        _lib().pe_device_autotune_log(self._h, buf, len(buf))
        return buf.value.decode()

    # diagnostics
    def trace_primary(self, camera: PerspectiveCamera, settings: RenderSettings, sample_index: int = 0,
                      ordered: bool = False):
        """Primary hit (shape, triangle within the shape, t) per pixel: through the 4-wide tree the
        render kernels use, or (ordered=True) the binary tree in the reference's visiting order."""
        n = settings.width * settings.height
        shape = np.empty(n, np.int32)
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        fn = _lib().pe_device_trace_primary_ordered if ordered else _lib().pe_device_trace_primary
        capi.check(fn(self._h, C.byref(camera.describe_gpu()), C.byref(settings.to_c()), sample_index,
                      capi.iptr(shape), capi.iptr(prim), capi.fptr(t)))
        return shape, prim, t

    def trace_rays(self, origins, directions, t_max, mode: int = 1, mask: int = VIS_ALL, time: float = 0.0):
        """Ray queries against the scene (a test probe): mode 0 closest hit on the binary tree in
        the reference's order, 1 closest hit on the 4-wide tree — (shape, prim, t), shape -1 on a
        miss — or 2 any hit — (occluded 0/1, -1, 0)."""
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        tm = np.ascontiguousarray(t_max, np.float32).reshape(-1)
        n = o.shape[0]
        shape = np.empty(n, np.int32)
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        capi.check(_lib().pe_device_trace_rays(self._h, capi.fptr(o), capi.fptr(d), capi.fptr(tm), n, int(mode), int(mask),
                                               float(time), capi.iptr(shape), capi.iptr(prim), capi.fptr(t)))
        return shape, prim, t

    def sobol(self, seed: int, px, py, index, n_dims: int) -> np.ndarray:
        px = np.ascontiguousarray(px, np.int32)
        py = np.ascontiguousarray(py, np.int32)
        index = np.ascontiguousarray(index, np.int32)
        out = np.empty((len(px), n_dims, 2), np.float32)
        capi.check(_lib().pe_device_sobol(self._h, seed, capi.iptr(px), capi.iptr(py), capi.iptr(index), len(px), n_dims,
                                          capi.fptr(out)))
        return out

    def bsdf_probe(self, material_index: int, queries) -> list:
        n = len(queries)
        q = (capi.pe_bsdf_query * n)(*queries)
        r = (capi.pe_bsdf_result * n)()
        capi.check(_lib().pe_device_bsdf_probe(self._h, material_index, q, n, r))
        return list(r)


def enumerate_devices() -> list[DeviceInfo]:
    out = [DeviceInfo(id="cpu", kind=DeviceKind.Cpu, name="host CPU", usable=False,
                      note="the CPU path is the reference engine's own; this build provides cuda:N only")]
    try:
        n = _lib().pe_device_count()
    except RuntimeError as e:
        out.append(DeviceInfo(id="cuda:0", kind=DeviceKind.Cuda, usable=False, note=str(e)))
        return out
    for i in range(n):
        out.append(DeviceInfo(id=f"cuda:{i}", kind=DeviceKind.Cuda, usable=True, note="B200 wavefront path tracer"))
    return out


def create_device(device_id: str = "auto", error: Optional[list] = None) -> Optional[CudaDevice]:
    """createDevice: ``cuda:N`` or ``auto``; returns None and appends the reason to ``error``."""
    try:
        if device_id in ("auto", "cuda"):
            ordinal = 0
        elif device_id.startswith("cuda:"):
            ordinal = int(device_id.split(":", 1)[1])
        else:
            raise ValueError(f"unknown device id '{device_id}' (this build serves cuda:N)")
        return CudaDevice(ordinal)
    except Exception as e:  # noqa: BLE001 — the reference reports, never throws
        if error is not None:
            error.append(str(e))
        return None


# ---------------------------------------------------------------------------------------------
@dataclasses.dataclass
class RequestStatus:
    state: int
    samples_done: int
    submit_ms: float
    start_ms: float
    done_ms: float
    paths: int
    error: int

    @property
    def done(self) -> bool:
        return self.state in (capi.PE_REQ_DONE, capi.PE_REQ_RELEASED)

    @property
    def latency_ms(self) -> float:
        return self.done_ms - self.submit_ms


class RenderServer:
    """Request server over one CudaDevice (pe_server_* in include/photon_cuda.h): resident scenes,
    device films admitted against an HBM budget, and continuous batching of many requests into
    shared waves.  A request's film equals a lone ``CudaDevice.render`` of samples [0, spp)."""

    def __init__(self, device: CudaDevice, budget_bytes: int):
        err = C.create_string_buffer(512)
        h = _lib().pe_server_create(device.handle, int(budget_bytes), err, len(err))
        if not h:
            raise capi.PhotonError(capi.PE_ERR_INVALID, err.value.decode())
        self._h = h
        self.device = device
        self._films = {}

    def close(self):
        if self._h:
            _lib().pe_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_scene(self, scene: Scene) -> int:
        if scene.info is None:
            scene.build_accelerator()
        sid = int(_lib().pe_server_add_scene(self._h, scene.handle))
        if sid < 0:
            capi.check(-sid)
        return sid

    def submit(self, scene_id: int, camera: PerspectiveCamera, settings: RenderSettings, spp: int,
               priority: int = 0) -> int:
        q = capi.pe_request_desc(scene_id, camera.describe_gpu(), settings.to_c(), int(spp), int(priority))
        rid = int(_lib().pe_server_submit(self._h, C.byref(q)))
        if rid < 0:
            capi.check(-rid)
        self._films[rid] = (settings.width, settings.height)
        return rid

    def status(self, rid: int) -> RequestStatus:
        st = capi.pe_request_status()
        capi.check(_lib().pe_server_status(self._h, rid, C.byref(st)))
        return RequestStatus(st.state, st.samples_done, st.submit_ms, st.start_ms, st.done_ms, st.paths, st.error)

    def wait(self, rid: int, timeout_ms: int = -1) -> bool:
        rc = _lib().pe_server_wait(self._h, rid, int(timeout_ms))
        if rc == capi.PE_ERR_CANCELLED:
            return False
        capi.check(rc)
        return True

    def take(self, rid: int) -> Film:
        w, h = self._films.pop(rid)
        f = Film(w, h)
        capi.check(_lib().pe_server_take(self._h, rid, capi.fptr(f.sum), capi.uptr(f.count), capi.fptr(f.sum_sq)))
        return f

    def stats(self) -> capi.pe_server_stats:
        s = capi.pe_server_stats()
        capi.check(_lib().pe_server_get_stats(self._h, C.byref(s)))
        return s


class RenderMode(enum.Enum):
    Interactive = 0
    Final = 1


@dataclasses.dataclass
class SessionConfig:
    mode: RenderMode = RenderMode.Final
    target_spp: int = 64
    time_limit: float = 0.0
    aovs: bool = False
    passes: bool = False
    batch_seconds: float = 0.5
    max_batch: int = 64


class RenderSession:
    """Batch policy over a device (src/engine/render_session.cpp:17-101)."""

    def __init__(self, device: CudaDevice):
        self.device = device
        self.camera = None
        self.film = Film()
        self.aovs: Optional[AovFilms] = None
        self.passes: Optional[RenderPassFilms] = None
        self.samples = 0
        self.traced = 0
        self._converged = False
        self.warnings: list[str] = []
        self._sps = 0.0
        self.last_batch_seconds = 0.0

    def begin(self, camera, settings: RenderSettings, config: SessionConfig):
        self.camera, self.settings, self.config = camera, dataclasses.replace(settings), dataclasses.replace(config)
        self.warnings = []
        f = self.device.features()
        name = self.device.info().name
        if self.config.aovs and not f.aovs:
            self.config.aovs = False
            self.warnings.append(f"{name}: AOVs are not supported; denoising uses colour only")
        if self.config.passes and not f.light_passes:
            self.config.passes = False
            self.warnings.append(f"{name}: render passes are not supported; beauty only")
        if self.settings.adaptive_sampling and not f.adaptive_sampling:
            self.settings.adaptive_sampling = False
            self.warnings.append(f"{name}: adaptive sampling is not supported; every pixel reaches the target")
        self.film.resize(max(1, settings.width), max(1, settings.height))
        self.aovs = AovFilms(max(1, settings.width), max(1, settings.height)) if self.config.aovs else None
        self.passes = RenderPassFilms(max(1, settings.width), max(1, settings.height)) if self.config.passes else None
        self.samples = 0
        self.traced = 0
        self._converged = False
        self._sps = 0.0
        self._start = time.perf_counter()

    def seconds(self) -> float:
        return time.perf_counter() - self._start

    def finished(self) -> bool:
        if self._converged:
            return True
        if self.config.target_spp > 0 and self.samples >= self.config.target_spp:
            return True
        return self.config.time_limit > 0.0 and self.samples > 0 and self.seconds() >= self.config.time_limit

    def next_batch(self) -> int:
        if self.config.mode == RenderMode.Interactive or self.samples == 0 or self._sps <= 0.0:
            return 1
        n = int(self.config.batch_seconds / self._sps)
        n = min(max(n, 1), max(1, self.config.max_batch))
        if self.config.target_spp > 0:
            n = min(n, self.config.target_spp - self.samples)
        if self.config.time_limit > 0.0:
            left = self.config.time_limit - self.seconds()
            n = min(n, max(1, int(left / self._sps)))
        return max(1, n)

    def advance(self, cancel=None) -> bool:
        if self.camera is None or self.finished():
            return False
        count = self.next_batch()
        t0 = time.perf_counter()
        r = self.device.render(self.camera, self.settings, RenderTargets(beauty=self.film, aovs=self.aovs, passes=self.passes), self.samples,
                               count, cancel)
        self.last_batch_seconds = time.perf_counter() - t0
        self.traced += r.samples_traced
        if not r.completed:
            return False
        self.samples += count
        per = self.last_batch_seconds / count
        self._sps = 0.5 * (self._sps + per) if self._sps > 0.0 else per
        # adaptive sampling: a batch that traced nothing means every pixel is clean
        # (render_session.cpp:99)
        if self.settings.adaptive_sampling and r.samples_traced == 0:
            self._converged = True
        return True

    def converged(self) -> bool:
        """RenderSession::converged: adaptive sampling left no pixel to sample."""
        return self._converged

    def average_samples(self) -> float:
        px = float(self.film.width * self.film.height)
        return self.traced / px if px > 0 else 0.0

    def resolve(self) -> np.ndarray:
        return self.film.resolve()


def rel_mse(x: np.ndarray, ref: np.ndarray) -> float:
    """relMSE = mean((x − ref)² / (ref² + 0.01)) over pixels and channels (scripts/compare_exr.py:30)."""
    x = x.astype(np.float64)
    ref = ref.astype(np.float64)
    return float(np.mean((x - ref) ** 2 / (ref * ref + 0.01)))
