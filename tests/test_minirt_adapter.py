"""The miniRT drop-in (libmrt_minirt.so): the reference's own t_minirt, as
its init_viewport builds it, rendered through the reference-named GPU entry
points (init_shader, convert_scene_build, convert_scene, compute_frame_gpu,
calc_one_sample, clean_*) and compared with the reference's CPU render of the
same structure: per pixel, from batch means of both renders (image-mean
bias, per-pixel z-scores and the bias relMSE, 42-minirt_b200/convergence.py)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class Vec3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


@pytest.fixture(scope="module")
def adapter(mrt, oracle):
    if not oracle.REF_LIB.exists():
        pytest.fail("oracle/_ref/liboracle_ref.so (the reference) is needed to build t_minirt")
    oracle.ref_lib()                        # reference symbols global first
    lib = C.CDLL(str(mrt.MINIRT_LIB_PATH))
    P = C.c_void_p
    for name, res, args in [("init_shader", C.c_int, [P, C.c_size_t, C.c_size_t, P]),
                            ("convert_scene_build", C.c_int, [P, P, P, P]),
                            ("convert_scene", None, [P, P, P, P]),
                            ("compute_frame_gpu", None, [P]),
                            ("calc_one_sample", None, [P, Vec3, C.c_int]),
                            ("clean_shaders", None, [P]), ("clean_scene", None, [P])]:
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


def gpu_batches(adapter, ref, m, n, batches):
    """compute_frame_gpu n times; batch means of the drop-in's float_render."""
    out, prev = [], ref.accum()
    for _ in range(batches):
        for _ in range(n // batches):
            adapter.compute_frame_gpu(m)
        cur = ref.accum()
        out.append((cur - prev) / (n // batches))
        prev = cur
    return np.stack(out)


def cpu_batches(ref, n, batches):
    """The reference's calc_one_sample n times; batch means."""
    out = []
    for _ in range(batches):
        ref.clear()
        ref.render(n // batches)
        out.append(ref.accum() / (n // batches))
    return np.stack(out)


def assert_same_image(gpu_bm, cpu_bm, what):
    """Per-pixel agreement of two independent renders of one scene, each
    given as batch means: no image-mean bias (4 standard errors per channel),
    at most 1 % of pixels beyond 5 standard errors (a shifted or blurred
    image fails at its edges), and the bias relMSE (both renders' noise
    subtracted) of the other pixels within 1e-3 plus 4 standard errors."""
    import convergence as cv
    g, r = cv.batch_summary(gpu_bm), cv.batch_summary(cpu_bm)
    st = cv.compare(g["mean"], g["var_mean"], g["batch_image_mean"], r)
    print(what, {k: st[k] for k in ("relmse_raw", "relmse_bias", "relmse_bias_se", "relmse_bias_inliers",
                                    "relmse_bias_inliers_se", "image_mean_z", "pixel_z_rms", "pixel_z_gt5")})
    assert np.all(np.abs(st["image_mean_z"]) <= 4.0), st
    assert st["pixel_z_gt5"] <= 0.01, st
    assert st["relmse_bias_inliers"] <= 1e-3 + 4 * st["relmse_bias_inliers_se"], st


def counters(ref):
    out = np.zeros(3, np.int32)
    ref.lib.refh_sample_counters(ref.h, out.ctypes.data)
    return out


def test_compute_frame_gpu_matches_reference_render(adapter, oracle, scenes):
    sc = scenes.make_c0(0, 48, 32, depth=8)
    ref = oracle.RefOracle(sc)
    L = ref.lib
    m, scn, vp = L.refh_minirt(ref.h), L.refh_scene_ptr(ref.h), L.refh_viewport_ptr(ref.h)
    sd, g = L.refh_shader_data(ref.h), L.refh_gpu_structs(ref.h)
    assert adapter.init_shader(sd, sc.width, sc.height, scn) == 0
    assert adapter.convert_scene_build(m, scn, vp, g) == 0
    cnt = np.zeros(6, np.int32)
    L.refh_gpu_counts(ref.h, cnt.ctypes.data)
    assert cnt[0] == 1 and cnt[1] == len(sc.spheres) and cnt[2] == len(sc.planes)
    adapter.convert_scene(m, scn, vp, g)
    n = 512
    gpu = gpu_batches(adapter, ref, m, n, 16)
    assert tuple(counters(ref)) == (n, n, n)
    # the reference itself, on a second copy of the same scene
    ref2 = oracle.RefOracle(sc)
    ref2.set_seed(2024)
    assert_same_image(gpu, cpu_batches(ref2, n, 16), "c0 drop-in")
    adapter.clean_shaders(sd)
    adapter.clean_scene(g)


def test_calc_one_sample_normals_mode_matches_reference(adapter, oracle, scenes):
    """render_mode 2 (first-hit normals) is deterministic: the drop-in
    calc_one_sample and the reference's give the same image for the same
    shared offset, and neither touches the sample counters."""
    sc = scenes.make_c1(1, 32, 24, depth=4, freq=8, sky=(32, 16))
    a, b = oracle.RefOracle(sc), oracle.RefOracle(sc)
    for r in (a, b):
        r.lib.refh_set_render_mode(r.h, 2)
    adapter.calc_one_sample(a.lib.refh_minirt(a.h), Vec3(0.25, 0.75, 0.0), 4)
    b.lib.refh_calc_one_sample(b.h, 0.25, 0.75, 4)
    ga, gb = a.accum(), b.accum()
    close = np.abs(ga - gb).max(axis=2) <= 1e-3
    assert close.mean() >= 0.995, close.mean()
    assert tuple(counters(a)) == (0, 0, 0)
    adapter.clean_shaders(a.lib.refh_shader_data(a.h))


def test_unsupported_objects_are_reported(adapter, oracle, scenes):
    sc = scenes.make_c0(0, 16, 16)
    ref = oracle.RefOracle(sc)
    L = ref.lib
    sd = L.refh_shader_data(ref.h)
    assert adapter.init_shader(sd, 16, 16, L.refh_scene_ptr(ref.h)) == 0
    adapter.clean_shaders(sd)
    # convert_scene_build without init_shader fails with -1 (and an [Error] line)
    assert adapter.convert_scene_build(L.refh_minirt(ref.h), L.refh_scene_ptr(ref.h),
                                       L.refh_viewport_ptr(ref.h), L.refh_gpu_structs(ref.h)) == -1


def test_compute_frame_gpu_with_quadrics_matches_reference_render(adapter, oracle, scenes):
    """Cylinders, cones and hyperboloids of t_scene go through the drop-in
    too: the image agrees with the reference's own CPU render per pixel."""
    sc = scenes.make_quadrics(5, 48, 36, depth=6)
    ref = oracle.RefOracle(sc)
    L = ref.lib
    m, scn, vp = L.refh_minirt(ref.h), L.refh_scene_ptr(ref.h), L.refh_viewport_ptr(ref.h)
    sd, g = L.refh_shader_data(ref.h), L.refh_gpu_structs(ref.h)
    assert adapter.init_shader(sd, sc.width, sc.height, scn) == 0
    assert adapter.convert_scene_build(m, scn, vp, g) == 0
    adapter.convert_scene(m, scn, vp, g)
    n = 512
    gpu = gpu_batches(adapter, ref, m, n, 16)
    ref2 = oracle.RefOracle(sc)
    ref2.set_seed(99)
    assert_same_image(gpu, cpu_batches(ref2, n, 16), "quadrics drop-in")
    adapter.clean_shaders(sd)
    adapter.clean_scene(g)


def test_compute_frame_gpu_with_textures_matches_reference_render(adapter, oracle, scenes):
    """t_tex images, checkers and maps of t_scene reach the drop-in."""
    sc = scenes.make_textured(6, 48, 36, depth=6)
    ref = oracle.RefOracle(sc)
    L = ref.lib
    m, scn, vp = L.refh_minirt(ref.h), L.refh_scene_ptr(ref.h), L.refh_viewport_ptr(ref.h)
    sd, g = L.refh_shader_data(ref.h), L.refh_gpu_structs(ref.h)
    assert adapter.init_shader(sd, sc.width, sc.height, scn) == 0
    assert adapter.convert_scene_build(m, scn, vp, g) == 0
    adapter.convert_scene(m, scn, vp, g)
    n = 512
    gpu = gpu_batches(adapter, ref, m, n, 16)
    ref2 = oracle.RefOracle(sc)
    ref2.set_seed(77)
    assert_same_image(gpu, cpu_batches(ref2, n, 16), "textures drop-in")
    adapter.clean_shaders(sd)
    adapter.clean_scene(g)
