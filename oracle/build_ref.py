"""CPU ORACLE - test infrastructure only: build the reference's own code.

Compiles files of the SolarEnergy_Chier reference tree (read in place from
/root/reference, never copied) with nvcc, straight from their sources, into
oracle/_ref/:

  libref_gpu.so    the reference's CUDA build (every source except main.cpp
                   and its tests) + ref/ref_gpu_shim.cu, for timing its
                   tracer on the GPU;
  libref_host.so   the reference's host code (scene files, configuration,
                   scene processing, grid cell lists, heliostat geometry,
                   3D-DDA, receiver intersection, energy, heap classes,
                   Buie tables, task files, flux-map text) + ref/ref_host_shim.cu,
                   linked against ref/host_cudart.cpp instead of libcudart,
                   so it runs on a machine without a GPU.

The reference's CMake build is not used (it needs the removed FindCUDA
module).  nlohmann/json.hpp, which the reference does not vendor, is taken
from the copy that ships inside the cudnn_frontend Python package of this
image (include path only).  oracle/_ref/ is git-ignored but travels with the
working tree, so machines without the reference tree use the prebuilt files.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
REF = Path(os.environ.get("QMCRT_REFERENCE_TREE", "/root/reference"))
NVCC = str(Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "bin" / "nvcc")

HOST_UNITS = [
    "Scene/SceneLoader.cpp", "Scene/SceneConfiguration.cpp", "Scene/SceneProcessor.cpp", "Scene/SolarScene.cpp",
    "Scene/SceneProcessor.cu",
    "Scene/DataStructure/Grid/Grid.cu", "Scene/DataStructure/Grid/RectangleGrid.cu",
    "Scene/DataStructure/Heliostat/Heliostat.cu", "Scene/DataStructure/Heliostat/RectangleHelio.cu",
    "Scene/DataStructure/Heliostat/FocusFlatRectangleHelio.cu",
    "Scene/DataStructure/Receiver/Receiver.cu", "Scene/DataStructure/Receiver/RectangleReceiver.cu",
    "Scene/DataStructure/Receiver/CylinderReceiver.cu", "Scene/DataStructure/Sunray/Sunray.cu",
    "QuasiMonteCarloRayTracing/Grid/rectGridDDA.cu",
    "Tool/FileLoader/RegularExpressionTree.cpp", "Tool/ImageSaver/ImageSaver.cpp",
    "RayTracingPipeline/TaskLoader.cpp",
]


def _json_include() -> Path | None:
    for p in sys.path:
        cand = Path(p) / "include" / "cudnn_frontend" / "thirdparty"
        if (cand / "nlohmann" / "json.hpp").exists():
            return cand
    return None


GPU_UNITS = HOST_UNITS + [
    "Scene/SceneProcessor.cu", "Tool/RandomNumberGenerator/RandomGenerator.cu",
    "Tool/RandomNumberGenerator/RandomGenerator.cpp",
    "QuasiMonteCarloRayTracing/QuasiMonteCarloRayTracer.cpp",
    "QuasiMonteCarloRayTracing/RectangleReceiverRectangleGridRayTracing.cu",
    "QuasiMonteCarloRayTracing/CylinderReceiverRectangleGridRayTracing.cu",
    "QuasiMonteCarloRayTracing/Receiver/rectangleReceiverIntersection.cu",
    "QuasiMonteCarloRayTracing/Receiver/cylinderReceiverIntersection.cu",
]


def include_flags() -> list[str]:
    dirs = ["Util", "Scene", "Scene/DataStructure/Grid", "Scene/DataStructure/Heliostat",
            "Scene/DataStructure/Receiver", "Scene/DataStructure/Sunray", "Tool", "QuasiMonteCarloRayTracing",
            "RayTracingPipeline", "."]
    flags = [f"-I{REF / d}" for d in dirs]
    j = _json_include()
    if j is not None:
        flags.append(f"-I{j}")
    return flags


def available() -> bool:
    return REF.exists() and (REF / "QuasiMonteCarloRayTracing").exists()


def build(force: bool = False) -> Path | None:
    lib = OUT / "libref_host.so"
    if not available():
        return lib if lib.exists() else None
    sources = [REF / u for u in HOST_UNITS] + [HERE / "ref" / "ref_host_shim.cu", HERE / "ref" / "host_cudart.cpp"]
    if not force and lib.exists() and all(lib.stat().st_mtime >= s.stat().st_mtime for s in sources):
        return lib
    obj_dir = OUT / "obj"
    obj_dir.mkdir(parents=True, exist_ok=True)
    common = ["-O2", "-std=c++14", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp", "-w",
              "-gencode", "arch=compute_100a,code=sm_100a"] + include_flags()
    objs = []
    for src in sources:
        obj = obj_dir / (src.stem + "_" + src.suffix[1:] + ".o")
        lang = ["-x", "cu"] if src.suffix == ".cu" else []
        cmd = [NVCC, *common, *lang, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"reference build failed on {src}")
        objs.append(str(obj))
    # -Bsymbolic: the reference code's CUDA runtime calls must bind to the host
    # stand-ins linked into this library even when another library in the
    # process (e.g. torch's libcudart) exports the same names globally.
    link = ["g++", "-shared", "-fopenmp", "-o", str(lib), *objs, "-Wl,--no-undefined", "-Wl,-Bsymbolic"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("reference link failed")
    return lib


def build_gpu(force: bool = False) -> Path | None:
    """libref_gpu.so: the reference's CUDA code as its own build would run it
    (-O3, sm_100a, relocatable device code, real CUDA runtime and cuRAND),
    plus ref/ref_gpu_shim.cu.  Used by bench.py to time the reference tracer."""
    lib = OUT / "libref_gpu.so"
    if not available():
        return lib if lib.exists() else None
    units = sorted(set(GPU_UNITS))
    sources = [REF / u for u in units] + [HERE / "ref" / "ref_gpu_shim.cu"]
    if not force and lib.exists() and all(lib.stat().st_mtime >= s.stat().st_mtime for s in sources):
        return lib
    obj_dir = OUT / "obj_gpu"
    obj_dir.mkdir(parents=True, exist_ok=True)
    common = ["-O3", "-std=c++14", "-rdc=true", "-Xcompiler", "-fPIC", "-w",
              "-gencode", "arch=compute_100a,code=sm_100a"] + include_flags()
    objs = []
    for src in sources:
        obj = obj_dir / (src.stem + "_" + src.suffix[1:] + ".o")
        lang = ["-x", "cu"]
        cmd = [NVCC, *common, *lang, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"reference GPU build failed on {src}")
        objs.append(str(obj))
    link = [NVCC, "-shared", "-rdc=true", "-gencode", "arch=compute_100a,code=sm_100a", "--cudart", "static",
            "-o", str(lib), *objs, "-lcurand"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("reference GPU link failed")
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
    print(build_gpu(force="--force" in sys.argv))
