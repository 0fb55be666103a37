"""Build recipe for the native libraries (run from anywhere).

  python 42-minirt_b200/build.py            -> 42-minirt_b200/libmrt.so
                                               (+ libmrt_minirt.so when the
                                               reference headers are present)

libmrt.so: CUDA C++ for sm_100a only, cudart linked statically so the library
depends on nothing but the driver. Built in-tree so it travels with the
repository snapshot. Translation units compile in parallel (one nvcc per
core); the megakernel instantiations are split per scene view type so that
no single unit dominates the build.

The miniRT headers that the drop-in adapter compiles against are looked up
in $MRT_REFERENCE_DIR/includes (default: the reference's mount point).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# (source, object stem, extra defines); longest first, so the parallel build
# starts the slow units first. render_inst.cu is compiled once per scene view
# type and kernel group (its header comment lists the groups).
_VIEWS = (("SceneViewT", "svt"), ("SceneViewQ", "svq"), ("SceneView", "sv"))
UNITS = [("render_inst.cu", f"render_{tag}_g{g}", [f"-DMRT_VIEW={view}", f"-DMRT_GROUP={g}"])
         for view, tag in _VIEWS for g in (0, 2, 3, 1)]
UNITS += [(src, Path(src).stem, []) for src in
          ("api.cu", "adjoint.cu", "wavefront.cu", "photon.cu", "render.cu", "readback.cu", "env.cu",
           "env_noalloc.cu", "bvh_build.cpp", "comm.cpp")]
REFERENCE_DIR = Path(os.environ.get("MRT_REFERENCE_DIR", "/root/reference"))


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_libmrt(verbose_ptxas: bool = False, jobs: int | None = None) -> Path:
    out = HERE / "libmrt.so"
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    objs, todo = [], []
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [INCLUDE / "mrt.h"]
    for src, stem, defines in UNITS:
        obj = objdir / (stem + ".o")
        objs.append(str(obj))
        path = CSRC / src
        deps = [path] + headers
        if obj.exists() and all(obj.stat().st_mtime >= d.stat().st_mtime for d in deps):
            continue
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
               "-I", str(CSRC), "-I", str(INCLUDE), *defines, "-c", str(path), "-o", str(obj)]
        if verbose_ptxas and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        todo.append(cmd)
    jobs = jobs or max(1, min(len(todo), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=jobs) as pool:
        for f in [pool.submit(_run, c) for c in todo]:
            f.result()
    stale = [o for o in objdir.glob("*.o") if str(o) not in objs]
    for o in stale:  # objects of units that no longer exist
        o.unlink()
    if todo or not out.exists():
        _run([NVCC, *ARCH, "-shared", "-o", str(out), *objs, "-lpthread", "-ldl"])
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


def build_minirt_adapter(minirt_includes: Path = REFERENCE_DIR / "includes") -> Path | None:
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
