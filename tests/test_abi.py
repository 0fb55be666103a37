"""The C-ABI boundary on the CPU: libmrt.so loads without a GPU, exports every
function include/mrt.h declares, the ctypes mirror has the C layouts, and
calls fail with the documented error codes instead of crashing."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
import tempfile
from pathlib import Path

import pytest

from conftest import REPO

HEADER = REPO / "include" / "mrt.h"


def declared_functions(header: Path) -> list[str]:
    return re.findall(r"^MRT_API\s+[\w\s\*]*?\**\s*(mrt_\w+)\(", header.read_text(), re.M)


def test_header_declares_the_boundary():
    names = declared_functions(HEADER)
    for need in ["mrt_create", "mrt_scene_build", "mrt_set_camera", "mrt_render", "mrt_read_accum",
                 "mrt_accumulate_double", "mrt_trace_first_hit", "mrt_destroy", "mrt_last_error"]:
        assert need in names


def test_library_loads_and_exports_every_declared_symbol(mrt):
    lib = mrt.load()
    out = subprocess.run(["nm", "-D", "--defined-only", str(mrt.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(\w+)", out))
    missing = [n for n in declared_functions(HEADER) if n not in exported]
    assert not missing, missing
    assert lib.mrt_version() == mrt.MRT_ABI_VERSION
    # nothing but the C-ABI leaks out of the library
    assert all(n.startswith("mrt_") or n.startswith("_") for n in exported), \
        sorted(n for n in exported if not n.startswith("mrt_"))[:10]


def test_ctypes_layouts_match_c(mrt):
    structs = {"mrt_material": mrt.Material, "mrt_sphere": mrt.Sphere, "mrt_plane": mrt.Plane,
               "mrt_mesh": mrt.Mesh, "mrt_cylinder": mrt.Cylinder, "mrt_cone": mrt.Cone,
               "mrt_hyperboloid": mrt.Hyperboloid, "mrt_texture": mrt.Texture, "mrt_light": mrt.Light, "mrt_camera": mrt.Camera,
               "mrt_ambient": mrt.Ambient, "mrt_caustic": mrt.Caustic,
               "mrt_scene_desc": mrt.SceneDesc, "mrt_render_params": mrt.RenderParams,
               "mrt_render_stats": mrt.RenderStats, "mrt_ray": mrt.Ray, "mrt_hit": mrt.Hit,
               "mrt_tune_entry": mrt.TuneEntry, "mrt_tune_result": mrt.TuneResult}
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"mrt.h\"\nint main(void){\n"
    for name in structs:
        src += f'  printf("{name} %zu\\n", sizeof({name}));\n'
    src += '  printf("off_scene_materials %zu\\n", offsetof(mrt_scene_desc, materials));\n'
    src += '  printf("off_scene_lights %zu\\n", offsetof(mrt_scene_desc, lights));\n'
    src += '  printf("off_scene_hyperboloids %zu\\n", offsetof(mrt_scene_desc, hyperboloids));\n'
    src += '  printf("off_scene_textures %zu\\n", offsetof(mrt_scene_desc, textures));\n'
    src += '  printf("off_mat_normal_intensity %zu\\n", offsetof(mrt_material, normal_intensity));\n'
    src += "  return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "sizes.c"
        c.write_text(src)
        exe = Path(d) / "sizes"
        subprocess.run(["gcc", "-I", str(REPO / "include"), str(c), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    got = dict(line.split() for line in out.strip().splitlines())
    for name, cls in structs.items():
        assert int(got[name]) == C.sizeof(cls), name
    assert int(got["off_scene_materials"]) == mrt.SceneDesc.materials.offset
    assert int(got["off_scene_lights"]) == mrt.SceneDesc.lights.offset
    assert int(got["off_scene_hyperboloids"]) == mrt.SceneDesc.hyperboloids.offset
    assert int(got["off_scene_textures"]) == mrt.SceneDesc.textures.offset
    assert int(got["off_mat_normal_intensity"]) == mrt.Material.normal_intensity.offset


def test_null_context_is_rejected_with_invalid(mrt):
    lib = mrt.load()
    assert lib.mrt_scene_build(None, None) == -1
    assert b"null" in lib.mrt_last_error()
    assert lib.mrt_render(None, None, None) == -1
    assert lib.mrt_trace_first_hit(None, None, 0, None) == -1
    lib.mrt_destroy(None)


def test_create_rejects_bad_sizes(mrt):
    lib = mrt.load()
    assert not lib.mrt_create(0, 0, 10)
    assert b"invalid render size" in lib.mrt_last_error()
    assert not lib.mrt_create(0, -5, 10)


def test_create_without_device_fails_loudly(mrt):
    lib = mrt.load()
    if lib.mrt_device_count() > 0:
        pytest.skip("a CUDA device is present")
    assert not lib.mrt_create(0, 64, 64)
    assert b"no CUDA device" in lib.mrt_last_error()
    with pytest.raises(mrt.MRTError):
        mrt.Context(64, 64)


def test_product_does_not_import_the_oracle():
    """The product path (the package) must never route through oracle/."""
    for f in (REPO / "42-minirt_b200").rglob("*.py"):
        txt = f.read_text()
        assert "import oracle" not in txt and "oracle/" not in txt.replace("# ", ""), f


def test_drop_in_exports_every_gpu_h_entry_point(mrt):
    """libmrt_minirt.so (the drop-in for miniRT's src/gpu) defines every
    function include/minirt_compat/gpu.h declares, gpu_bvh_sah included
    (read from the dynamic symbol table; nothing is loaded)."""
    import re
    import shutil
    lib = Path(mrt.MINIRT_LIB_PATH)
    if not lib.exists():
        pytest.skip("libmrt_minirt.so is built only where the reference headers are present")
    nm = shutil.which("nm")
    assert nm, "binutils nm is needed"
    decl = (REPO / "include" / "minirt_compat" / "gpu.h").read_text()
    names = set(re.findall(r"^\w[\w\s\*]*?\b(\w+)\(", decl, re.M))
    assert {"init_shader", "convert_scene_build", "compute_frame_gpu", "gpu_bvh_sah"} <= names
    out = subprocess.run([nm, "-D", "--defined-only", str(lib)], capture_output=True, text=True, check=True).stdout
    defined = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert names <= defined, sorted(names - defined)
