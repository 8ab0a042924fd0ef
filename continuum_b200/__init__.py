"""B200-native mask-cone area-light visibility (Continuum's hot path).

The product is libcontinuum_cuda.so (hand-written sm_100a CUDA behind a C
ABI, include/continuum_cuda.h); this package binds it and mirrors the
reference's visibility API.
"""
from .kernel import (Batch, Hierarchy, Light, LightingCache, MaskConeKernel, PageRequest, Planner, RectLight, Scene,
                     Server, SphereLight, Spot, Visibility, flatten_meshes, host_scene, host_scene_instanced, light_gpu,
                     lights_gpu, receivers_gpu)

__all__ = [
    "Batch", "Hierarchy", "Light", "LightingCache", "MaskConeKernel", "PageRequest", "Planner", "RectLight", "Scene",
    "Server", "SphereLight", "Spot", "Visibility",
    "flatten_meshes", "host_scene", "host_scene_instanced", "light_gpu", "lights_gpu", "receivers_gpu",
]
