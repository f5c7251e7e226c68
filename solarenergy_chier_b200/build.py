"""In-tree build of the native library and the drop-in executable.

Produces, next to this file:
  libqmcrt.so   the C ABI of include/qmcrt.h (host C++ + sm_100a kernels)
  bin/qmcrt     the RayTracingPipeline command-line executable

Host C++ is compiled by g++ with -ffp-contract=off so that the scene
geometry rounds exactly as the reference's host code does.  The tracer is
compiled twice: with FMA contraction (production) and with -fmad=false (every
float operation rounded like the CPU oracle).  Only nvcc and g++ are needed;
the build works on a machine without a GPU.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
OBJ = PKG / "_build"
LIB = PKG / "libqmcrt.so"
EXE = PKG / "bin" / "qmcrt"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")

HOST_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-ffp-contract=off"] + ARCH

HOST_SOURCES = ["scene.cpp", "buie_table.cpp", "capi.cpp", "batch.cpp", "diff.cpp", "pipeline.cpp"]
CUDA_UNITS = [
    ("tracer.cu", "tracer_fast.o", ["-DQM_TRACE_VARIANT=fast", "-DQM_TRACE_THREADS=32", "-DQM_TRACE_MIN_BLOCKS=28",
                                       "-DQM_TRACE_FAST_DIVIDE", "-DQM_TRACE_CANDIDATE_HITS"]),
    ("tracer.cu", "tracer_fast4.o", ["-DQM_TRACE_VARIANT=fast4", "-DQM_TRACE_MIN_BLOCKS=4", "-DQM_TRACE_FAST_DIVIDE",
                                        "-DQM_TRACE_CANDIDATE_HITS"]),
    ("tracer.cu", "tracer_exact.o", ["-DQM_TRACE_VARIANT=exact", "-DQM_TRACE_THREADS=32", "-DQM_TRACE_MIN_BLOCKS=28",
                                        "-DQM_EXACT_ACOS", "-fmad=false"]),
    # launch shapes of the production build timed by the autotuner (qmcrt_autotune):
    # warp chunks of 32 or 128 iterations, two-warp blocks
    ("tracer.cu", "tracer_fast_c32.o", ["-DQM_TRACE_VARIANT=fast_c32", "-DQM_TRACE_THREADS=32", "-DQM_TRACE_MIN_BLOCKS=28",
                                           "-DQM_CHUNK_ITERS=32", "-DQM_TRACE_FAST_DIVIDE", "-DQM_TRACE_CANDIDATE_HITS"]),
    ("tracer.cu", "tracer_fast_c128.o", ["-DQM_TRACE_VARIANT=fast_c128", "-DQM_TRACE_THREADS=32",
                                            "-DQM_TRACE_MIN_BLOCKS=28", "-DQM_CHUNK_ITERS=128", "-DQM_TRACE_FAST_DIVIDE",
                                            "-DQM_TRACE_CANDIDATE_HITS"]),
    ("tracer.cu", "tracer_fast_ps.o", ["-DQM_TRACE_VARIANT=fast_ps", "-DQM_TRACE_THREADS=32", "-DQM_TRACE_MIN_BLOCKS=28",
                                          "-DQM_TRACE_FAST_DIVIDE", "-DQM_TRACE_CANDIDATE_HITS", "-DQM_TRACE_PERSISTENT"]),
    ("tracer.cu", "tracer_fast_t64.o", ["-DQM_TRACE_VARIANT=fast_t64", "-DQM_TRACE_THREADS=64", "-DQM_TRACE_MIN_BLOCKS=14",
                                           "-DQM_TRACE_FAST_DIVIDE", "-DQM_TRACE_CANDIDATE_HITS"]),
    ("tracer.cu", "tracer_rx.o", ["-DQM_TRACE_VARIANT=rx", "-DQM_TRACE_THREADS=32", "-DQM_TRACE_MIN_BLOCKS=28",
                                     "-DQM_TRACE_FAST_DIVIDE", "-DQM_TRACE_CANDIDATE_HITS", "-DQM_TRACE_APPROX_RECEIVER"]),
    ("tracer.cu", "tracer_approx.o", ["-DQM_TRACE_VARIANT=approx", "-DQM_TRACE_THREADS=32", "-DQM_TRACE_MIN_BLOCKS=28",
                                         "-DQM_TRACE_FAST_DIVIDE", "-DQM_TRACE_CANDIDATE_HITS", "-DQM_TRACE_APPROX_MATH"]),
    ("pools.cu", "pools.o", []),
    ("power.cu", "power.o", []),
    # per-sun preparation: no FMA contraction, so it matches the host geometry bit for bit
    ("prep.cu", "prep.o", ["-fmad=false"]),
    ("diff.cu", "diff_kernels.o", []),
    ("grid_build.cu", "grid_build.o", ["-fmad=false"]),
    ("smooth.cu", "smooth.o", []),
    ("microbench.cu", "microbench.o", []),
    ("smooth_static.cu", "smooth_static.o", []),
]


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def _digest(paths: list[Path], extra: list[str]) -> str:
    h = hashlib.sha256()
    for p in paths:
        h.update(p.read_bytes())
    h.update(" ".join(extra).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every unit whose inputs changed and link libqmcrt.so and bin/qmcrt."""
    OBJ.mkdir(exist_ok=True)
    EXE.parent.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))
    objects = []
    for src in HOST_SOURCES:
        obj = OBJ / (Path(src).stem + ".o")
        cmd = ["g++", *HOST_FLAGS, f"-I{CSRC}", f"-I{INCLUDE}", f"-I{CUDA_HOME / 'include'}", "-c",
               str(CSRC / src), "-o", str(obj)]
        _compile(obj, [CSRC / src, *headers], cmd, force, verbose)
        objects.append(obj)
    for src, name, flags in CUDA_UNITS:
        obj = OBJ / name
        cmd = [NVCC, *NVCC_FLAGS, *flags, f"-I{CSRC}", f"-I{INCLUDE}", "-c", str(CSRC / src), "-o", str(obj)]
        _compile(obj, [CSRC / src, *headers], cmd, force, verbose)
        objects.append(obj)
    # The CUDA runtime is linked statically: the library does not depend on
    # whichever libcudart.so.12 another package (e.g. torch) loaded first.
    link = [NVCC, *ARCH, "-shared", "--cudart", "static", "-o", str(LIB), *map(str, objects)]
    _link(LIB, objects, link, force, verbose)
    main_obj = OBJ / "main.o"
    _compile(main_obj, [CSRC / "main.cpp", INCLUDE / "qmcrt.h"],
             ["g++", *HOST_FLAGS, f"-I{INCLUDE}", "-c", str(CSRC / "main.cpp"), "-o", str(main_obj)], force, verbose)
    _link(EXE, [main_obj, LIB], ["g++", "-o", str(EXE), str(main_obj), f"-L{PKG}", "-lqmcrt",
                                  "-Wl,-rpath,$ORIGIN/.."], force, verbose)
    return LIB


def _compile(obj: Path, inputs: list[Path], cmd: list[str], force: bool, verbose: bool) -> None:
    stamp = obj.with_suffix(obj.suffix + ".sha")
    digest = _digest(inputs, cmd)
    if not force and obj.exists() and stamp.exists() and stamp.read_text() == digest:
        return
    if verbose:
        print(" ".join(cmd))
    _run(cmd)
    stamp.write_text(digest)


def _link(out: Path, inputs: list[Path], cmd: list[str], force: bool, verbose: bool) -> None:
    if not force and out.exists() and all(out.stat().st_mtime >= p.stat().st_mtime for p in inputs):
        return
    if verbose:
        print(" ".join(cmd))
    _run(cmd)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
