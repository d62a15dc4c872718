"""spectral_b200: B200-native spectral path tracing behind the reference's render API.

Drop-in for the Taichi kernels of Xyzonox/taichi-spectral-render main.py: the
scene stays a ``create_scene()`` dictionary, the render loop keeps its
cast_rays / average_and_reset_block / color_rays / clear_pixel_space cadence,
and every kernel is hand-written CUDA for sm_100a in libspectral.so, reached
through a C ABI (include/spectral.h).
"""
from . import _lib
from ._lib import SpectralError, build, load
from .renderer import RenderConfig, Renderer, fov_scale_for
from .scene import (F32_KEYS, I32_KEYS, PROP_ANISTROPY_FACTOR, PROP_EMISSION, PROP_EXTINCTION_COEFFICIENT,
                    PROP_IS_TRUE_VOLUME, PROP_REFRACTIVE_INDEX, PROP_ROUGHNESS, PROP_SCATTERING_COEFFICIENT,
                    PROP_SURFACE_EMISSION, compile_scene, flatten_triangles, get_scene_dimensions, material_tables)

__all__ = ["Renderer", "RenderConfig", "SpectralError", "build", "load", "compile_scene", "flatten_triangles",
           "get_scene_dimensions", "material_tables", "fov_scale_for"]
