"""B200-native transient path tracer: the GPU drop-in for the reference renderer's
``TransientRenderer::render`` (LeksiDor/JaraboTransientRendering).

The compute path is libtransient_b200.so (CUDA, sm_100a) behind the C ABI of
include/transient_b200.h; this package is its host-side binding.
"""
from . import scenes
from .renderer import (Context, Batch, Guide, World, Lambertian, GGX, PointLightSource, RectangularAreaLightSource,
                       HenyeyGreenstein, HomogeneousMedium, PinholeCamera, StreakCameraFilm, MultibounceStreakFilm,
                       StratifiedSampler, BidirectionalPathTracing, TransientRenderer, HIT_DTYPE, INVALID_ID)
from ._abi import TransientError, LIB_PATH

__all__ = ["scenes", "Context", "Batch", "Guide", "World", "Lambertian", "GGX", "PointLightSource", "RectangularAreaLightSource",
           "HenyeyGreenstein", "HomogeneousMedium", "PinholeCamera", "StreakCameraFilm", "MultibounceStreakFilm", "StratifiedSampler",
           "BidirectionalPathTracing", "TransientRenderer", "TransientError", "HIT_DTYPE", "INVALID_ID",
           "LIB_PATH"]
