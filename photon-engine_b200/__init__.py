"""photon-engine_b200 — B200-native (sm_100a) path-tracing device for the photon engine's render API.

The product is ``libphoton_cuda.so`` (C ABI in ``include/photon_cuda.h``); this package is the
host-side mirror of the reference's RenderDevice / RenderSession / Scene API over it.
"""
from . import _capi
from .engine import (VIS_ALL, VIS_CAMERA, VIS_DIFFUSE, VIS_GLOSSY, VIS_SHADOW, VIS_TRANSMISSION, AovFilms, AreaLight, Background, BackgroundMode, CudaDevice, Dielectric, DeviceFeatures, DeviceInfo,
                     DisneyMaterial, EnvironmentLight, Film, Lambertian, LightPass, Material, MeshInstance, Mirror, OrthographicCamera, PerspectiveCamera, ThinLensCamera,
                     PixelFilterType, RenderMode, RenderPassFilms, RenderServer, RenderSession, RenderSettings, RenderTargets, RequestStatus,
                     SampleBatchResult,
                     Scene, SceneUpdateKind, SessionConfig, Sphere, TriangleMesh, create_device, enumerate_devices, rel_mse)

__all__ = [n for n in dir() if not n.startswith("_")] + ["_capi"]
