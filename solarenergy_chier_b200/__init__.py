"""B200-native quasi-Monte-Carlo heliostat-field ray tracer.

A drop-in for the QuasiMonteCarloRayTracer path of SolarEnergy_Chier: the
native library libqmcrt.so (C ABI in include/qmcrt.h, sm_100a kernels in
csrc/) does all the work; this package is its Python binding.
"""
from ._lib import LIB_PATH, QmcrtError, load  # noqa: F401
from .scene import (  # noqa: F401
    SUNSHAPE_BUIE,
    Batch,
    Diff,
    SUNSHAPE_PILLBOX,
    ImageSaver,
    ImageSmoother,
    QuasiMonteCarloRayTracer,
    RayTracingPipeline,
    Scene,
    executable,
    launch_shapes,
    pipeline_run,
    save_text,
    smooth_device,
)

__all__ = [
    "Scene", "Batch", "Diff", "QuasiMonteCarloRayTracer", "ImageSmoother", "ImageSaver", "RayTracingPipeline",
    "SUNSHAPE_BUIE", "SUNSHAPE_PILLBOX", "QmcrtError", "load", "LIB_PATH", "save_text", "smooth_device",
    "pipeline_run", "executable", "launch_shapes",
]
