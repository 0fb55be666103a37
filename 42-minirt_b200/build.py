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
SOURCES = ["api.cu", "render.cu", "readback.cu", "wavefront.cu", "env.cu", "env_noalloc.cu", "photon.cu", "adjoint.cu",
           "bvh_build.cpp"]


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


def minirt_overlay(minirt_includes: Path) -> Path:
    """Header overlay for compiling against miniRT: links to miniRT's own
    includes/*.h, except its GL bridge headers (gpu.h, gpu_struct.h,
    gpu_scene.h), which resolve to include/minirt_compat."""
    ov = HERE / "_build" / "minirt_overlay"
    ov.mkdir(parents=True, exist_ok=True)
    compat = INCLUDE / "minirt_compat"
    for h in sorted(minirt_includes.glob("*.h")):
        target = compat / h.name if (compat / h.name).exists() else h
        link = ov / h.name
        if link.is_symlink() or link.exists():
            link.unlink()
        link.symlink_to(target)
    return ov


def build_minirt_adapter(minirt_includes: Path = Path("/root/reference/includes")) -> Path | None:
    """libmrt_minirt.so: miniRT's GPU entry points (init_shader,
    convert_scene_build, convert_scene, compute_frame_gpu, calc_one_sample,
    clean_*) compiled against miniRT's own headers. Needs the miniRT
    includes directory; without it the prebuilt library is kept."""
    out = HERE / "libmrt_minirt.so"
    src = HERE / "minirt" / "minirt_gpu.c"
    if not minirt_includes.exists():
        return out if out.exists() else None
    if out.exists() and out.stat().st_mtime >= max(src.stat().st_mtime,
                                                     (HERE / "libmrt.so").stat().st_mtime):
        return out
    ov = minirt_overlay(minirt_includes)
    _run(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu99", "-w", "-I", str(ov),
          "-I", str(HERE / "minirt" / "headless"), "-I", str(INCLUDE), str(src),
          "-o", str(out), "-L", str(HERE), "-lmrt", "-Wl,-rpath,$ORIGIN"])
    return out


def main() -> int:
    build_libmrt(verbose_ptxas="-v" in sys.argv)
    build_minirt_adapter()
    return 0


if __name__ == "__main__":
    sys.exit(main())
