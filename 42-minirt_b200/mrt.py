"""ctypes mirror of include/mrt.h and a thin Python handle over libmrt.so.

The library is the product; this module only declares the C structs and
function signatures so that tests, the benchmark and Python users can call the
C-ABI directly. There is no Python fallback: if libmrt.so is missing or cannot
be loaded, every entry point raises.

Struct layouts follow include/mrt.h field for field (ctypes applies the same
natural alignment as the C compiler on x86-64).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libmrt.so"
MINIRT_LIB_PATH = HERE / "libmrt_minirt.so"

MRT_ABI_VERSION = 4

MRT_OK = 0
STATUS_NAMES = {
    0: "MRT_OK", -1: "MRT_ERR_INVALID", -2: "MRT_ERR_CUDA", -3: "MRT_ERR_OOM",
    -4: "MRT_ERR_QUEUE_OVERFLOW", -5: "MRT_ERR_BUDGET", -6: "MRT_ERR_ABORTED",
    -7: "MRT_ERR_NO_DEVICE", -8: "MRT_ERR_STACK",
}

FORM_MEGAKERNEL, FORM_WAVEFRONT, FORM_AUTO, FORM_MEGAKERNEL_PLAIN = 0, 1, 2, 3
JITTER_SHARED, JITTER_PIXEL = 0, 1
LIGHT_POINT, LIGHT_DIRECTIONAL = 0, 1

u8x3 = C.c_uint8 * 3
f64x3 = C.c_double * 3
f32x3 = C.c_float * 3


TEX_IMAGE, TEX_HDR, TEX_COLOR, TEX_CHECKER_LOCAL, TEX_CHECKER_GLOBAL = range(5)
TEX_SLOTS = ["color_tex", "metallic_tex", "roughness_tex", "transmission_tex", "ao_tex",
             "emission_strength_tex", "emission_color_tex", "normal_tex"]


class Texture(C.Structure):
    _fields_ = [("type", C.c_int32), ("width", C.c_uint32), ("height", C.c_uint32),
                ("pad_", C.c_int32), ("rgba", C.POINTER(C.c_uint8)), ("checker_scale", C.c_double),
                ("c1", u8x3), ("c2", u8x3), ("pad2_", C.c_uint8 * 2)]


class Material(C.Structure):
    _fields_ = [("color", u8x3), ("emission_color", u8x3), ("pad_", C.c_uint8 * 2),
                ("metallic", C.c_double), ("roughness", C.c_double), ("ior", C.c_double),
                ("transmission", C.c_double), ("ao", C.c_double),
                ("emission_strength", C.c_double), ("scale", C.c_double)] + \
        [(k, C.c_int32) for k in TEX_SLOTS] + [("normal_intensity", C.c_double)]


class Sphere(C.Structure):
    _fields_ = [("center", f64x3), ("radius", C.c_double), ("material", C.c_int32),
                ("color", u8x3), ("pad_", C.c_uint8)]


class Plane(C.Structure):
    _fields_ = [("point", f64x3), ("normal", f64x3), ("material", C.c_int32),
                ("color", u8x3), ("pad_", C.c_uint8)]


class Cylinder(C.Structure):
    _fields_ = [("position", f64x3), ("orientation", f64x3), ("diameter", C.c_double),
                ("height", C.c_double), ("material", C.c_int32), ("material_top", C.c_int32),
                ("material_bot", C.c_int32), ("color", u8x3), ("pad_", C.c_uint8)]


class Cone(C.Structure):
    _fields_ = [("position", f64x3), ("orientation", f64x3), ("diameter", C.c_double),
                ("height", C.c_double), ("material", C.c_int32), ("material_top", C.c_int32),
                ("color", u8x3), ("pad_", C.c_uint8 * 5)]


class Hyperboloid(C.Structure):
    _fields_ = [("position", f64x3), ("orientation", f64x3), ("a", C.c_double),
                ("b", C.c_double), ("c", C.c_double), ("shape", C.c_double),
                ("height", C.c_double), ("material", C.c_int32), ("color", u8x3),
                ("pad_", C.c_uint8)]


class Mesh(C.Structure):
    _fields_ = [("n_vertices", C.c_uint32), ("n_triangles", C.c_uint32),
                ("positions", C.POINTER(C.c_double)), ("normals", C.POINTER(C.c_double)),
                ("uvs", C.POINTER(C.c_double)), ("indices", C.POINTER(C.c_uint32)),
                ("tri_material", C.POINTER(C.c_int32)), ("material", C.c_int32),
                ("color", u8x3), ("pad_", C.c_uint8)]


class Light(C.Structure):
    _fields_ = [("type", C.c_int32), ("shadow_sample", C.c_int32), ("position", f64x3),
                ("brightness", C.c_double), ("radius", C.c_float), ("color", u8x3),
                ("pad_", C.c_uint8)]


class Camera(C.Structure):
    _fields_ = [("position", f64x3), ("orientation", f64x3), ("focus_dist", C.c_double),
                ("defocus_angle", C.c_double), ("fov", C.c_uint8), ("pad_", C.c_uint8 * 7)]


class Ambient(C.Structure):
    _fields_ = [("ratio", C.c_double), ("hdr_rgbe", C.POINTER(C.c_uint8)),
                ("hdr_width", C.c_int32), ("hdr_height", C.c_int32),
                ("hdr_exposure", C.c_float), ("hdr_gamma", C.c_float),
                ("color", u8x3), ("pad_", C.c_uint8 * 5)]


class Caustic(C.Structure):
    _fields_ = [("enable", C.c_int32), ("passes", C.c_int32),
                ("photons_per_light", C.c_uint64), ("radius", C.c_double),
                ("norm_factor", C.c_double), ("shrink", C.c_double),
                ("knn", C.c_int32), ("mode", C.c_int32), ("spp_per_pass", C.c_int32),
                ("pad_", C.c_int32)]


class SceneDesc(C.Structure):
    _fields_ = [("abi_version", C.c_uint32), ("render_width", C.c_int32),
                ("render_height", C.c_int32), ("max_bounces", C.c_int32),
                ("triangle_one_sided", C.c_int32), ("pad_", C.c_int32),
                ("ior_all", C.c_double), ("camera", Camera), ("ambient", Ambient),
                ("caustic", Caustic),
                ("materials", C.POINTER(Material)), ("n_materials", C.c_int32),
                ("n_spheres", C.c_int32), ("spheres", C.POINTER(Sphere)),
                ("planes", C.POINTER(Plane)), ("n_planes", C.c_int32),
                ("n_meshes", C.c_int32), ("meshes", C.POINTER(Mesh)),
                ("lights", C.POINTER(Light)), ("n_lights", C.c_int32),
                ("pad2_", C.c_int32),
                ("cylinders", C.POINTER(Cylinder)), ("cones", C.POINTER(Cone)),
                ("hyperboloids", C.POINTER(Hyperboloid)), ("n_cylinders", C.c_int32),
                ("n_cones", C.c_int32), ("n_hyperboloids", C.c_int32), ("n_textures", C.c_int32),
                ("textures", C.POINTER(Texture))]


class RenderParams(C.Structure):
    _fields_ = [("spp", C.c_int32), ("sample_base", C.c_int32), ("seed", C.c_uint64),
                ("max_bounces", C.c_int32), ("form", C.c_int32), ("jitter", C.c_int32),
                ("render_mode", C.c_int32), ("block_size", C.c_int32),
                ("queue_capacity", C.c_int32), ("sort_threshold", C.c_int32),
                ("use_graph", C.c_int32), ("env_sampler", C.c_int32),
                ("offset", C.POINTER(C.c_double))]


class RenderStats(C.Structure):
    _fields_ = [("ms", C.c_double), ("paths", C.c_uint64), ("segments", C.c_uint64),
                ("shadow_rays", C.c_uint64), ("kernel_launches", C.c_uint32),
                ("status", C.c_int32)]


class TuneEntry(C.Structure):
    _fields_ = [("form", C.c_int32), ("block_size", C.c_int32), ("queue_capacity", C.c_int32),
                ("sort_threshold", C.c_int32), ("mpaths_s", C.c_double)]


class TuneResult(C.Structure):
    _fields_ = [("n", C.c_int32), ("best", C.c_int32), ("entry", TuneEntry * 32)]


class BvhOptions(C.Structure):
    _fields_ = [("mode", C.c_int32), ("pad_", C.c_int32), ("n_prims", C.c_int64),
                ("order", C.POINTER(C.c_int32)), ("positions", C.POINTER(C.c_double))]


BVH_SAH, BVH_REFERENCE, BVH_WIDE = 0, 1, 2


class Ray(C.Structure):
    _fields_ = [("orig", f64x3), ("dir", f64x3)]


class Hit(C.Structure):
    _fields_ = [("prim", C.c_int32), ("front_face", C.c_int32), ("t", C.c_float),
                ("u", C.c_float), ("v", C.c_float), ("normal", f32x3), ("point", f32x3),
                ("visits", C.c_int32)]


HIT_DTYPE = np.dtype([("prim", "<i4"), ("front_face", "<i4"), ("t", "<f4"), ("u", "<f4"),
                      ("v", "<f4"), ("normal", "<f4", 3), ("point", "<f4", 3),
                      ("visits", "<i4")])
assert HIT_DTYPE.itemsize == C.sizeof(Hit)

_P = C.c_void_p

SIGNATURES = {
    "mrt_last_error": (C.c_char_p, []),
    "mrt_version": (C.c_int, []),
    "mrt_device_count": (C.c_int, []),
    "mrt_create": (_P, [C.c_int, C.c_int, C.c_int]),
    "mrt_destroy": (None, [_P]),
    "mrt_scene_build": (C.c_int, [_P, C.POINTER(SceneDesc)]),
    "mrt_set_camera": (C.c_int, [_P, C.POINTER(Camera), C.c_double, C.c_double]),
    "mrt_render": (C.c_int, [_P, C.POINTER(RenderParams), C.POINTER(RenderStats)]),
    "mrt_clear": (C.c_int, [_P]),
    "mrt_render_batch": (C.c_int, [C.POINTER(_P), C.POINTER(RenderParams), C.c_int32,
                                   C.POINTER(RenderStats)]),
    "mrt_tune": (C.c_int, [_P, C.c_int32, C.c_uint64, C.POINTER(TuneResult)]),
    "mrt_read_accum": (C.c_int, [_P, _P, C.POINTER(C.c_int32)]),
    "mrt_accumulate_double": (C.c_int, [_P, _P]),
    "mrt_read_depth": (C.c_int, [_P, _P]),
    "mrt_render_state_save": (C.c_int, [_P, C.c_char_p]),
    "mrt_render_state_load": (C.c_int, [_P, C.c_char_p]),
    "mrt_comm_unique_id": (C.c_int, [_P]),
    "mrt_set_bvh_options": (C.c_int, [_P, _P]),
    "mrt_read_bvh_leaves": (C.c_int64, [_P, _P, C.c_int64]),
    "mrt_bvh_build_check": (C.c_int, [_P, C.c_int64, C.c_int32, _P]),
    "mrt_comm_init": (C.c_int, [_P, _P, C.c_int32, C.c_int32]),
    "mrt_reduce_frame": (C.c_int, [_P, C.c_int32]),
    "mrt_comm_destroy": (C.c_int, [_P]),
    "mrt_shard_samples": (None, [C.c_int64, C.c_int32, C.c_int32, _P, _P]),
    "mrt_trace_first_hit": (C.c_int, [_P, _P, C.c_int64, _P]),
    "mrt_trace_paths": (C.c_int, [_P, C.POINTER(RenderParams), _P, _P, C.c_int32, _P, _P]),
    "mrt_read_env_tables": (C.c_int, [_P, _P, _P, _P]),
    "mrt_env_sample": (C.c_int, [_P, C.c_int64, C.c_uint64, C.c_int32, _P, _P]),
    "mrt_photon_count": (C.c_int64, [_P]),
    "mrt_read_photons": (C.c_int, [_P, _P, _P, C.c_int64]),
    "mrt_set_photons": (C.c_int, [_P, _P, _P, C.c_int64]),
    "mrt_caustic_query": (C.c_int, [_P, _P, C.c_int64, C.c_int32, _P]),
    "mrt_env_tables_noalloc": (C.c_int, [C.c_int, _P, C.c_int32, C.c_int32, C.c_float, _P, _P, _P, _P]),
    "mrt_diff_layout": (C.c_int64, [_P, C.POINTER(C.c_int64)]),
    "mrt_diff_get_params": (C.c_int, [_P, _P]),
    "mrt_forward": (C.c_int, [_P, _P, C.POINTER(RenderParams), _P, C.POINTER(RenderStats)]),
    "mrt_backward": (C.c_int, [_P, _P, C.POINTER(RenderParams), _P, _P, C.POINTER(RenderStats)]),
}


class MRTError(RuntimeError):
    pass


def render_batch(ctxs: list, params: list[dict], block_size: int = 0) -> "RenderStats":
    """One call over the scenes of several contexts (same device): megakernel
    scenes in one persistent launch per view type, wavefront scenes each in
    its own wavefront, all on concurrent streams. params[i]["form"] picks the
    form per scene (FORM_AUTO: the scene's tuned choice)."""
    lib = load()
    n = len(ctxs)
    arr = (_P * n)(*[c.h for c in ctxs])
    ps = (RenderParams * n)()
    for i, p in enumerate(params):
        ps[i] = RenderParams(spp=p["spp"], sample_base=p.get("sample_base", 0), seed=p.get("seed", 1),
                             max_bounces=p.get("max_bounces", 0), jitter=p.get("jitter", 0),
                             env_sampler=p.get("env_sampler", 0), block_size=block_size,
                             form=p.get("form", FORM_MEGAKERNEL))
    st = RenderStats()
    check(lib.mrt_render_batch(arr, ps, n, C.byref(st)), "mrt_render_batch")
    return st


_lib = None

COMM_ID_BYTES = 128


def bvh_build_check(boxes, mode: int = BVH_WIDE) -> dict:
    """mrt_bvh_build_check: build the BVH over (n, 6) boxes (min xyz, max
    xyz) on the host and check the wide tree's structure."""
    b = np.ascontiguousarray(boxes, np.float64).reshape(-1, 6)
    st = np.zeros(4, np.int64)
    check(load().mrt_bvh_build_check(_ptr(b), len(b), mode, _ptr(st)), "mrt_bvh_build_check")
    return {"nodes": int(st[0]), "depth": int(st[1]), "leaves": int(st[2]), "wide": bool(st[3])}


def comm_unique_id() -> bytes:
    """A new NCCL communicator id (mrt_comm_unique_id), to be sent to every rank."""
    buf = (C.c_ubyte * COMM_ID_BYTES)()
    check(load().mrt_comm_unique_id(buf), "mrt_comm_unique_id")
    return bytes(buf)


def shard_samples(total: int, world: int, rank: int) -> tuple[int, int]:
    """(first, count) of rank's contiguous sample shard (mrt_shard_samples)."""
    first, count = C.c_int64(), C.c_int64()
    load().mrt_shard_samples(total, world, rank, C.byref(first), C.byref(count))
    return first.value, count.value


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load libmrt.so (built in-tree by build.py). Raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise MRTError(f"{p} not built: run `python 42-minirt_b200/build.py` "
                       "(or __graft_entry__.build())")
    lib = C.CDLL(str(p), mode=C.RTLD_GLOBAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(rc: int, what: str) -> None:
    if rc != MRT_OK:
        msg = load().mrt_last_error()
        raise MRTError(f"{what} failed: {STATUS_NAMES.get(rc, rc)}: "
                       f"{msg.decode() if msg else ''}")


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _buf(a, what: str):
    """Pointer of a contiguous float32 numpy array (host) or torch tensor
    (host or this context's GPU): the differentiable entry points take both."""
    if hasattr(a, "data_ptr"):
        if str(a.dtype) != "torch.float32" or not a.is_contiguous():
            raise MRTError(f"{what}: needs a contiguous float32 tensor")
        return C.c_void_p(a.data_ptr())
    if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous):
        raise MRTError(f"{what}: needs a C-contiguous float32 array")
    return _ptr(a)


class Context:
    """One device context (mrt_ctx): scene + accumulator on one GPU."""

    def __init__(self, width: int, height: int, device: int = 0):
        self.lib = load()
        self.width, self.height = int(width), int(height)
        self.h = self.lib.mrt_create(int(device), self.width, self.height)
        if not self.h:
            raise MRTError(f"mrt_create failed: {self.lib.mrt_last_error().decode()}")
        self._keep = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.mrt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build(self, scene) -> None:
        desc = scene.desc() if hasattr(scene, "desc") else scene
        self._keep = scene
        check(self.lib.mrt_scene_build(self.h, C.byref(desc)), "mrt_scene_build")

    def set_camera(self, cam: Camera, ior_all: float, ratio: float) -> None:
        check(self.lib.mrt_set_camera(self.h, C.byref(cam), ior_all, ratio), "mrt_set_camera")

    def render(self, spp: int, seed: int = 1, sample_base: int = 0, form: int = FORM_MEGAKERNEL,
               jitter: int = JITTER_SHARED, max_bounces: int = 0, render_mode: int = 0,
               block_size: int = 0, queue_capacity: int = 0, sort_threshold: int = 0,
               use_graph: int = 0, env_sampler: int = 0, offset=None) -> RenderStats:
        p = RenderParams(spp=spp, sample_base=sample_base, seed=seed, max_bounces=max_bounces,
                         form=form, jitter=jitter, render_mode=render_mode,
                         block_size=block_size, queue_capacity=queue_capacity,
                         sort_threshold=sort_threshold, use_graph=use_graph,
                         env_sampler=env_sampler)
        off = None
        if offset is not None:
            off = (C.c_double * 2)(float(offset[0]), float(offset[1]))
            p.offset = C.cast(off, C.POINTER(C.c_double))
        st = RenderStats()
        check(self.lib.mrt_render(self.h, C.byref(p), C.byref(st)), "mrt_render")
        return st

    def tune(self, spp: int = 2, seed: int = 1) -> list[dict]:
        """Times the forms / launch shapes, keeps the fastest for FORM_AUTO."""
        r = TuneResult()
        check(self.lib.mrt_tune(self.h, spp, seed, C.byref(r)), "mrt_tune")
        names = {FORM_MEGAKERNEL: "megakernel", FORM_WAVEFRONT: "wavefront",
                 FORM_MEGAKERNEL_PLAIN: "megakernel_plain"}
        return [dict(form=names[e.form], block_size=e.block_size, queue_capacity=e.queue_capacity,
                     sort_threshold=e.sort_threshold, mpaths_s=e.mpaths_s, best=(i == r.best))
                for i, e in enumerate(r.entry[:r.n])]

    def clear(self) -> None:
        check(self.lib.mrt_clear(self.h), "mrt_clear")

    def read_accum(self) -> tuple[np.ndarray, int]:
        out = np.zeros((self.height, self.width, 3), np.float32)
        spp = C.c_int32(0)
        check(self.lib.mrt_read_accum(self.h, _ptr(out), C.byref(spp)), "mrt_read_accum")
        return out, spp.value

    def accumulate_double(self, buf: np.ndarray) -> None:
        assert buf.dtype == np.float64 and buf.size == self.width * self.height * 3
        check(self.lib.mrt_accumulate_double(self.h, _ptr(buf)), "mrt_accumulate_double")

    def save_state(self, path) -> None:
        check(self.lib.mrt_render_state_save(self.h, str(path).encode()), "mrt_render_state_save")

    def load_state(self, path) -> None:
        check(self.lib.mrt_render_state_load(self.h, str(path).encode()), "mrt_render_state_load")

    # multi-GPU sample sharding (one process per GPU, NCCL)
    def comm_init(self, comm_id: bytes, rank: int, world: int) -> None:
        """Joins the communicator made by comm_unique_id() on one rank."""
        assert len(comm_id) == COMM_ID_BYTES
        buf = (C.c_ubyte * COMM_ID_BYTES).from_buffer_copy(comm_id)
        check(self.lib.mrt_comm_init(self.h, buf, rank, world), "mrt_comm_init")

    def reduce_frame(self, root: int = 0) -> None:
        """Sums every rank's accumulator and sample count into root's."""
        check(self.lib.mrt_reduce_frame(self.h, root), "mrt_reduce_frame")

    def comm_destroy(self) -> None:
        check(self.lib.mrt_comm_destroy(self.h), "mrt_comm_destroy")

    def set_bvh_options(self, mode: int, order=None, positions=None) -> None:
        """BVH build for the next build(): BVH_SAH (default, the binary SAH
        tree), BVH_WIDE (the 8-wide tree, for scenes without quadrics or
        textures) or BVH_REFERENCE (the
        reference's median-split tree, traversed left first, with the
        reference's node-visit count in render_mode 1). order: flat ids in the
        reference's object-list order; positions: (n, 3) split positions."""
        o = BvhOptions(mode=mode)
        keep = []
        if order is not None:
            a = np.ascontiguousarray(order, np.int32)
            keep.append(a)
            o.order = a.ctypes.data_as(C.POINTER(C.c_int32))
            o.n_prims = len(a)
        if positions is not None:
            b = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
            keep.append(b)
            o.positions = b.ctypes.data_as(C.POINTER(C.c_double))
            o.n_prims = len(b)
        check(self.lib.mrt_set_bvh_options(self.h, C.byref(o)), "mrt_set_bvh_options")

    def bvh_leaves(self) -> np.ndarray:
        """Flat primitive ids in leaf order (mrt_read_bvh_leaves)."""
        n = self.lib.mrt_read_bvh_leaves(self.h, None, 0)
        if n < 0:
            check(int(n), "mrt_read_bvh_leaves")
        out = np.zeros(max(1, n), np.int32)
        self.lib.mrt_read_bvh_leaves(self.h, _ptr(out), n)
        return out[:n]

    def read_depth(self) -> np.ndarray:
        out = np.zeros((self.height, self.width), np.int32)
        check(self.lib.mrt_read_depth(self.h, _ptr(out)), "mrt_read_depth")
        return out

    def first_hit(self, orig: np.ndarray, dirs: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(np.concatenate([orig, dirs], axis=1), np.float64)
        hits = np.zeros(len(rays), HIT_DTYPE)
        check(self.lib.mrt_trace_first_hit(self.h, _ptr(rays), len(rays), _ptr(hits)),
              "mrt_trace_first_hit")
        return hits

    def trace_paths(self, pixels, samples, seed: int = 1, jitter: int = JITTER_SHARED,
                    env_sampler: int = 1, max_bounces: int = 0):
        """Per-bounce event records (n, 16, 20) and radiance (n, 3) of single paths."""
        pix = np.ascontiguousarray(pixels, np.int32)
        smp = np.ascontiguousarray(samples, np.int32)
        ev = np.zeros((len(pix), 16, 20), np.float32)
        rgb = np.zeros((len(pix), 3), np.float32)
        p = RenderParams(seed=seed, jitter=jitter, env_sampler=env_sampler, max_bounces=max_bounces)
        check(self.lib.mrt_trace_paths(self.h, C.byref(p), _ptr(pix), _ptr(smp), len(pix),
                                       _ptr(ev), _ptr(rgb)), "mrt_trace_paths")
        return ev, rgb

    def env_tables(self, w: int, h: int):
        pdf = np.zeros(w * h, np.float32)
        cm = np.zeros(h, np.float32)
        cc = np.zeros(w * h, np.float32)
        check(self.lib.mrt_read_env_tables(self.h, _ptr(pdf), _ptr(cm), _ptr(cc)),
              "mrt_read_env_tables")
        return pdf, cm, cc

    def env_sample(self, n: int, seed: int = 1, sampler: int = 0):
        """(outcome index, float4 dir+pdf) of n importance samples."""
        out = np.zeros((n, 4), np.float32)
        k = np.zeros(n, np.int32)
        check(self.lib.mrt_env_sample(self.h, n, seed, sampler, _ptr(k), _ptr(out)),
              "mrt_env_sample")
        return k, out

    def photon_count(self) -> int:
        n = self.lib.mrt_photon_count(self.h)
        if n < 0:
            check(int(n), "mrt_photon_count")
        return int(n)

    def photons(self):
        n = self.photon_count()
        pos = np.zeros((n, 4), np.float32)
        pw = np.zeros((n, 4), np.float32)
        check(self.lib.mrt_read_photons(self.h, _ptr(pos), _ptr(pw), n), "mrt_read_photons")
        return pos[:, :3], pw[:, :3]

    def set_photons(self, pos: np.ndarray, power: np.ndarray) -> None:
        pos = np.ascontiguousarray(pos, np.float64)
        power = np.ascontiguousarray(power, np.float64)
        check(self.lib.mrt_set_photons(self.h, _ptr(pos), _ptr(power), len(pos)),
              "mrt_set_photons")

    def caustic_query(self, pts: np.ndarray, k: int = 15) -> np.ndarray:
        pts = np.ascontiguousarray(pts, np.float64)
        out = np.zeros((len(pts), 3), np.float64)
        check(self.lib.mrt_caustic_query(self.h, _ptr(pts), len(pts), k, _ptr(out)),
              "mrt_caustic_query")
        return out

    # -------------------------------------------- differentiable rendering

    def diff_layout(self) -> dict:
        """Sizes of the theta blocks: albedo (M*3), roughness (M), emission
        (M), sky (H*W*3), in that order."""
        c = (C.c_int64 * 4)()
        n = self.lib.mrt_diff_layout(self.h, c)
        if n < 0:
            check(int(n), "mrt_diff_layout")
        return {"albedo": c[0], "roughness": c[1], "emission": c[2], "sky": c[3], "total": int(n)}

    def diff_params(self) -> np.ndarray:
        """theta of the scene as built."""
        out = np.zeros(self.diff_layout()["total"], np.float32)
        check(self.lib.mrt_diff_get_params(self.h, _ptr(out)), "mrt_diff_get_params")
        return out

    @staticmethod
    def _diff_params(spp, seed, sample_base, max_bounces, jitter) -> RenderParams:
        return RenderParams(spp=spp, sample_base=sample_base, seed=seed, max_bounces=max_bounces,
                            jitter=jitter)

    def forward(self, theta, spp: int, seed: int = 1, sample_base: int = 0, max_bounces: int = 0,
                jitter: int = JITTER_SHARED, out=None, stats: bool = False):
        """Image (H, W, 3) float32, the mean of `spp` samples, rendered with
        parameters theta. `out` may be a float32 numpy array or torch tensor
        (host or device) of H*W*3 elements."""
        if out is None:
            out = np.zeros((self.height, self.width, 3), np.float32)
        st = RenderStats()
        p = self._diff_params(spp, seed, sample_base, max_bounces, jitter)
        check(self.lib.mrt_forward(self.h, _buf(theta, "theta"), C.byref(p), _buf(out, "image"),
                                   C.byref(st)), "mrt_forward")
        return (out, st) if stats else out

    def backward(self, theta, grad_image, spp: int, seed: int = 1, sample_base: int = 0,
                 max_bounces: int = 0, jitter: int = JITTER_SHARED, out=None, stats: bool = False):
        """d loss / d theta for d loss / d image, replaying the forward's paths
        (same theta, spp, seed, sample_base, max_bounces, jitter)."""
        if out is None:
            out = np.zeros(self.diff_layout()["total"], np.float32)
        st = RenderStats()
        p = self._diff_params(spp, seed, sample_base, max_bounces, jitter)
        check(self.lib.mrt_backward(self.h, _buf(theta, "theta"), C.byref(p),
                                    _buf(grad_image, "grad_image"), _buf(out, "grad_theta"),
                                    C.byref(st)), "mrt_backward")
        return (out, st) if stats else out



# ------------------------------------------------ render_state.rts (host side)

def write_rts(path, float_render: np.ndarray, sample: int) -> None:
    """render_state.rts as export_render_state writes it
    (export_render_state.c:15-33): int32 width, height, sample, then the
    (H, W, 3) double per-pixel sums, little-endian."""
    fr = np.ascontiguousarray(float_render, "<f8")
    h, w = fr.shape[:2]
    with open(path, "wb") as f:
        f.write(np.array([w, h, sample], "<i4").tobytes())
        f.write(fr.tobytes())


def read_rts(path) -> tuple[np.ndarray, int]:
    """(float_render (H, W, 3) float64, sample) of a render_state.rts, with
    init_float_render's size check (export_render_state.c:35-51)."""
    raw = open(path, "rb").read()
    if len(raw) < 12:
        raise ValueError(f"{path}: no header")
    w, h, sample = (int(x) for x in np.frombuffer(raw[:12], "<i4"))
    if len(raw) - 12 != w * h * 3 * 8:
        raise ValueError(f"{path}: {len(raw) - 12} data bytes for a {w}x{h} render")
    return np.frombuffer(raw[12:], "<f8").reshape(h, w, 3).copy(), sample
