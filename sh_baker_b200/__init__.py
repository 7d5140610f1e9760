"""B200-native SH9 lightmap bake: the hot path of sh-baker (UV raster ->
BVH -> path tracing with NEE -> SH9 -> downsample -> dilation) as CUDA
kernels for sm_100a behind a C ABI (include/shb.h)."""
from .api import (BakeConfig, BakeResult, BakeSHLightMap, Context, CreateValidityMask, DeviceScene, Dilate,
                  DownsampleEnvironmentVisibilityTexture, DownsampleSHTexture, DownsampleValidityMask,
                  FindOcclusion, GBuffer, RasterConfig, RasterizeScene, default_context, rasterize_to_device)
from .scene import (AREA, DIRECTIONAL, POINT, SPOT, SURFACE_POINT_DTYPE, Geometry, Light, Material, Scene,
                    Texture, pack_scene)

__all__ = [
    "BakeConfig", "BakeResult", "BakeSHLightMap", "Context", "CreateValidityMask", "DeviceScene", "Dilate",
    "DownsampleEnvironmentVisibilityTexture", "DownsampleSHTexture", "DownsampleValidityMask", "FindOcclusion",
    "GBuffer", "RasterConfig", "RasterizeScene", "default_context", "rasterize_to_device", "AREA", "DIRECTIONAL",
    "POINT", "SPOT", "SURFACE_POINT_DTYPE", "Geometry", "Light", "Material", "Scene", "Texture", "pack_scene",
]
