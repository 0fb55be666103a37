"""Build recipe for the native libraries (run from anywhere).

  python 42-minirt_b200/build.py            -> 42-minirt_b200/libmrt.so
                                               (+ libmrt_minirt.so when the
                                               reference headers are present)

libmrt.so: CUDA C++ for sm_100a only, cudart linked statically so the library
depends on nothing but the driver. Built in-tree so it travels with the
repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["api.cu", "render.cu", "wavefront.cu", "env.cu", "photon.cu", "bvh_build.cpp"]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_libmrt(verbose_ptxas: bool = False) -> Path:
    out = HERE / "libmrt.so"
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        objs.append(str(obj))
        path = CSRC / src
        deps = [path] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [INCLUDE / "mrt.h"]
        if obj.exists() and all(obj.stat().st_mtime >= d.stat().st_mtime for d in deps):
            continue
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
               "-I", str(CSRC), "-I", str(INCLUDE), "-c", str(path), "-o", str(obj)]
        if verbose_ptxas and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        _run(cmd)
    _run([NVCC, *ARCH, "-shared", "-o", str(out), *objs, "-lpthread"])
    return out


def build_minirt_adapter() -> Path | None:
    """libmrt_minirt.so: the reference-named entry points (init_shader,
    convert_scene_build, compute_frame_gpu, calc_one_sample, ...) compiled
    against miniRT's own headers (overlaid with include/minirt_compat)."""
    overlay = HERE.parent / "oracle" / "_ref" / "overlay"
    if not overlay.exists():
        return None
    out = HERE / "libmrt_minirt.so"
    src = HERE / "minirt" / "minirt_gpu.c"
    if not src.exists():
        return None
    if out.exists() and out.stat().st_mtime >= max(src.stat().st_mtime,
                                                     (HERE / "libmrt.so").stat().st_mtime):
        return out
    _run(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu99", "-w", "-I", str(overlay),
          "-I", str(HERE.parent / "oracle" / "shim"), "-I", str(INCLUDE), str(src),
          "-o", str(out), "-L", str(HERE), "-lmrt", "-Wl,-rpath,$ORIGIN"])
    return out


def main() -> int:
    build_libmrt(verbose_ptxas="-v" in sys.argv)
    build_minirt_adapter()
    return 0


if __name__ == "__main__":
    sys.exit(main())
