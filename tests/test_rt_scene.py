"""A .rt scene file end to end: the reference's own parser (parse_scene,
compiled from its sources into oracle/_ref with stand-ins for its
un-vendored libft) builds t_scene; the reference renders it on the CPU and
the drop-in (convert_scene_build + compute_frame_gpu) renders the same
t_scene on the GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import GOLDEN

RT = GOLDEN / "parse_scene.rt"


def test_reference_parser_reads_the_scene(oracle, has_reference):
    if not has_reference:
        pytest.skip("reference not built here (oracle/_ref)")
    ref = oracle.RefOracle.from_rt(RT, 32, 24, 4)
    oracle.ref_lib().refh_set_seed(3)
    ref.render(2)
    img = ref.accum()
    assert np.isfinite(img).all() and img.mean() > 0.05
    ref.close()


class Vec3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


@pytest.mark.gpu
def test_drop_in_renders_the_parsed_scene_like_the_reference(mrt, oracle):
    if not oracle.REF_LIB.exists():
        pytest.fail("oracle/_ref/liboracle_ref.so (the reference) is needed to parse .rt files")
    oracle.ref_lib()
    lib = C.CDLL(str(mrt.MINIRT_LIB_PATH))
    P = C.c_void_p
    for name, res, args in [("init_shader", C.c_int, [P, C.c_size_t, C.c_size_t, P]),
                            ("convert_scene_build", C.c_int, [P, P, P, P]),
                            ("convert_scene", None, [P, P, P, P]),
                            ("compute_frame_gpu", None, [P]),
                            ("clean_shaders", None, [P]), ("clean_scene", None, [P])]:
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    W, H, depth, n = 48, 36, 6, 512
    ref = oracle.RefOracle.from_rt(RT, W, H, depth)
    L = ref.lib
    m, scn, vp = L.refh_minirt(ref.h), L.refh_scene_ptr(ref.h), L.refh_viewport_ptr(ref.h)
    sd, g = L.refh_shader_data(ref.h), L.refh_gpu_structs(ref.h)
    assert lib.init_shader(sd, W, H, scn) == 0
    assert lib.convert_scene_build(m, scn, vp, g) == 0
    lib.convert_scene(m, scn, vp, g)
    from test_minirt_adapter import assert_same_image, cpu_batches, gpu_batches
    gpu = gpu_batches(lib, ref, m, n, 16)
    cpu_ref = oracle.RefOracle.from_rt(RT, W, H, depth)
    cpu_ref.set_seed(11)
    assert_same_image(gpu, cpu_batches(cpu_ref, n, 16), "parsed .rt scene")
    lib.clean_shaders(sd)
    lib.clean_scene(g)
