"""mrt_env_tables_noalloc: the HDRI table build for hosts that cannot
allocate GPU memory when they need the tables (all device memory comes from
their own arena or pool, or the calling loop must never reach the
allocator). The caller passes device buffers for the sky and the three
tables; the build's scratch is a fixed array inside the library.

Checked against the tables of the ordinary path (mrt_scene_build, read back
with mrt_read_env_tables), bit for bit as the other table tests do, on two
calls in a row with different skies, so that what the first call leaves in
the shared scratch cannot leak into the second. The file name sorts last so
that a run stopping at the first failure has run every other test before it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sky_scene(scenes, w, h, seed, exposure):
    sc = scenes.make_c4(width=32, height=32, spp=1, depth=2, freq=4, n_materials=2, sky=(w, h))
    sc.hdr = scenes.make_sky(w, h, seed)
    sc.hdr_exposure = exposure
    return sc


def _reference_tables(mrt, oracle, sc):
    ctx = mrt.Context(sc.width, sc.height)
    ctx.build(oracle.canonical_scene(sc))
    h, w = sc.hdr.shape[:2]
    out = ctx.env_tables(w, h)
    ctx.close()
    return out


def _noalloc(lib, torch, sc):
    h, w = sc.hdr.shape[:2]
    rgbe = torch.tensor(np.ascontiguousarray(sc.hdr, np.uint8).reshape(-1), device="cuda")
    pdf = torch.full((w * h,), -1.0, device="cuda")
    cm = torch.full((h,), -1.0, device="cuda")
    cc = torch.full((w * h,), -1.0, device="cuda")
    torch.cuda.synchronize()
    rc = lib.mrt_env_tables_noalloc(0, C.c_void_p(rgbe.data_ptr()), w, h, float(sc.hdr_exposure),
                                    C.c_void_p(pdf.data_ptr()), C.c_void_p(cm.data_ptr()),
                                    C.c_void_p(cc.data_ptr()), None)
    assert rc == 0, lib.mrt_last_error().decode()
    return pdf.cpu().numpy(), cm.cpu().numpy(), cc.cpu().numpy()


def test_noalloc_tables_match_the_scene_build(mrt, scenes, oracle):
    torch = pytest.importorskip("torch")
    lib = mrt.load()
    assert lib.mrt_device_count() > 0, "gpu tests need a CUDA device"
    skies = [_sky_scene(scenes, 512, 256, 21, 0.0), _sky_scene(scenes, 256, 128, 22, 0.5)]
    refs = [_reference_tables(mrt, oracle, sc) for sc in skies]
    for call, (sc, ref) in enumerate(zip(skies, refs)):
        free_before = torch.cuda.mem_get_info()[0]
        got = _noalloc(lib, torch, sc)
        if call > 0:   # after the first call's set-up nothing more is reserved
            assert torch.cuda.mem_get_info()[0] >= free_before - (2 << 20)
        for g, r in zip(got, ref):
            np.testing.assert_array_equal(g, r)


def test_noalloc_rejects_a_sky_beyond_its_scratch(mrt):
    torch = pytest.importorskip("torch")
    lib = mrt.load()
    buf = torch.zeros(16, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    w, h = 1024, 512   # 524,288 texels > MRT_ENV_NOALLOC_MAX_TEXELS
    rc = lib.mrt_env_tables_noalloc(0, p, w, h, 0.0, p, p, p, None)
    assert rc == -1   # MRT_ERR_INVALID
    assert "exceeds the fixed scratch" in lib.mrt_last_error().decode()
    rc = lib.mrt_env_tables_noalloc(0, p, 1, 64, 0.0, p, p, p, None)
    assert rc == -1   # MRT_ERR_INVALID
