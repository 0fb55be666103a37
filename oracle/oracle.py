"""TEST INFRASTRUCTURE — ctypes access to the two CPU oracles.

 * RefOracle: the reference's own CPU path (miniRT C sources compiled by
   oracle/Makefile into oracle/_ref/liboracle_ref.so), driven through
   oracle/ref_harness.c.
 * Restatement: this project's FP64 C restatement of the same algorithms
   (oracle/mrt_oracle.c -> oracle/libmrt_oracle.so), which adds the per-path
   counter-based RNG used by the CUDA kernels so single paths can be compared.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this module, and only as the checker / the timed CPU reference — never as a
product path.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
sys.path.insert(0, str(REPO / "42-minirt_b200"))
import mrt  # noqa: E402

REF_LIB = HERE / "_ref" / "liboracle_ref.so"
RST_LIB = HERE / "libmrt_oracle.so"

REF_HIT_DTYPE = np.dtype([("prim", "<i4"), ("front_face", "<i4"), ("depth", "<i4"),
                          ("pad_", "<i4"), ("t", "<f8"), ("u", "<f8"), ("v", "<f8"),
                          ("point", "<f8", 3), ("normal", "<f8", 3), ("color", "<f8", 3)])

_P = C.c_void_p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


_ref = None


def ref_lib():
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle ref)")
        lib = C.CDLL(str(REF_LIB), mode=C.RTLD_GLOBAL)
        sig = {
            "refh_create": (_P, [_P]), "refh_destroy": (None, [_P]),
            "refh_create_from_rt": (_P, [C.c_char_p, C.c_int, C.c_int, C.c_int]),
            "refh_set_seed": (None, [C.c_uint64]), "refh_get_seed": (C.c_uint64, []),
            "refh_set_quiet": (None, [C.c_int]), "refh_random_double": (C.c_double, []),
            "refh_first_hit": (C.c_int, [_P, _P, C.c_int64, _P]),
            "refh_path_trace": (C.c_int, [_P, _P, C.c_int, _P]),
            "refh_render": (C.c_int, [_P, C.c_int, _P]),
            "refh_render_pixels": (C.c_int, [_P, _P, C.c_int64, C.c_int]),
            "refh_set_render_mode": (C.c_int, [_P, C.c_int]),
            "refh_float_render": (C.POINTER(C.c_double), [_P]),
            "refh_depth_buffer": (C.POINTER(C.c_int), [_P]),
            "refh_clear": (None, [_P]), "refh_viewport": (None, [_P, _P]),
            "refh_triangle_positions": (C.c_int, [_P, _P]),
            "refh_bvh": (C.c_int, [_P, _P, _P, _P]),
            "refh_object_list": (C.c_int, [_P, _P, _P]),
            "refh_env_tables": (C.c_int, [_P, _P, _P, _P, _P]),
            "refh_env_sample": (C.c_int, [_P, C.c_int64, _P, _P]),
            "refh_background": (C.c_int, [_P, _P, C.c_int64, C.c_int, _P]),
            "refh_photon_count": (C.c_int64, [_P]),
            "refh_photons": (C.c_int, [_P, _P, _P, _P]),
            "refh_caustic_query": (C.c_int, [_P, _P, C.c_int64, C.c_int, _P]),
            "refh_minirt": (_P, [_P]), "refh_scene_ptr": (_P, [_P]),
            "refh_viewport_ptr": (_P, [_P]), "refh_shader_data": (_P, [_P]),
            "refh_gpu_structs": (_P, [_P]), "refh_sample_counters": (C.c_int, [_P, _P]),
            "refh_gpu_counts": (C.c_int, [_P, _P]),
            "refh_calc_one_sample": (None, [_P, C.c_double, C.c_double, C.c_int]),
        }
        for k, (r, a) in sig.items():
            f = getattr(lib, k)
            f.restype, f.argtypes = r, a
        lib.refh_set_quiet(1)
        _ref = lib
    return _ref


class RefOracle:
    """The reference's CPU renderer on one flat scene."""

    def __init__(self, scene):
        self.lib = ref_lib()
        self.scene = scene
        self.desc = scene.desc()
        self.h = self.lib.refh_create(C.byref(self.desc))
        if not self.h:
            raise ValueError("refh_create rejected the scene")
        self.W, self.H = scene.width, scene.height

    @classmethod
    def from_rt(cls, path, width: int, height: int, max_bounces: int):
        """A .rt scene file through the reference's own parser."""
        self = cls.__new__(cls)
        self.lib = ref_lib()
        self.scene, self.desc = None, None
        self.h = self.lib.refh_create_from_rt(str(path).encode(), width, height, max_bounces)
        if not self.h:
            raise ValueError(f"the reference's parser rejected {path}")
        self.W, self.H = width, height
        return self

    def close(self):
        if self.h:
            self.lib.refh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_seed(self, seed: int):
        self.lib.refh_set_seed(seed)

    def first_hit(self, orig, dirs):
        rays = np.ascontiguousarray(np.concatenate([orig, dirs], 1), np.float64)
        out = np.zeros(len(rays), REF_HIT_DTYPE)
        self.lib.refh_first_hit(self.h, _ptr(rays), len(rays), _ptr(out))
        return out

    def path_trace(self, orig, d, max_depth):
        ray = np.ascontiguousarray(np.concatenate([orig, d]), np.float64)
        out = np.zeros(3)
        self.lib.refh_path_trace(self.h, _ptr(ray), max_depth, _ptr(out))
        return out

    def render(self, spp: int):
        offs = np.zeros((spp, 3))
        self.lib.refh_render(self.h, spp, _ptr(offs))
        return offs

    def render_pixels(self, pix: np.ndarray, spp: int):
        pix = np.ascontiguousarray(pix, np.int32)
        self.lib.refh_render_pixels(self.h, _ptr(pix), len(pix), spp)

    def accum(self) -> np.ndarray:
        p = self.lib.refh_float_render(self.h)
        return np.ctypeslib.as_array(p, shape=(self.H, self.W, 3)).copy()

    def clear(self):
        self.lib.refh_clear(self.h)

    def viewport(self):
        out = np.zeros(12)
        self.lib.refh_viewport(self.h, _ptr(out))
        return dict(pixel00=out[0:3], du=out[3:6], dv=out[6:9], cam=out[9:12])

    def triangle_positions(self):
        n = self.scene.n_triangles
        out = np.zeros((n, 9))
        self.lib.refh_triangle_positions(self.h, _ptr(out))
        return out

    def bvh(self):
        n_prims = self.scene.n_prims_bvh()
        nn = max(1, 2 * n_prims)
        b = np.zeros((nn, 6))
        info = np.zeros((nn, 5), np.uint32)
        prim = np.zeros(max(1, n_prims), np.int32)
        n = self.lib.refh_bvh(self.h, _ptr(b), _ptr(info), _ptr(prim))
        return b[:n], info[:n], prim[:n_prims]

    def object_list(self):
        """The reference's BVH object list: flat ids in its order, and each
        entry's split position (get_obj_position)."""
        n = self.scene.n_prims_bvh()
        flat = np.zeros(max(1, n), np.int32)
        pos = np.zeros((max(1, n), 3))
        k = self.lib.refh_object_list(self.h, _ptr(flat), _ptr(pos))
        return flat[:k], pos[:k]

    def env_tables(self):
        if self.scene.hdr is None:
            return None
        h, w = self.scene.hdr.shape[:2]
        pdf = np.zeros(w * h, np.float32)
        cm = np.zeros(h, np.float32)
        cc = np.zeros(w * h, np.float32)
        avg = C.c_double(0)
        ok = self.lib.refh_env_tables(self.h, _ptr(pdf), _ptr(cm), _ptr(cc), C.byref(avg))
        return (pdf, cm, cc, avg.value) if ok else None

    def env_sample(self, n: int):
        uv = np.zeros((n, 2))
        d = np.zeros((n, 3))
        self.lib.refh_env_sample(self.h, n, _ptr(uv), _ptr(d))
        return uv, d

    def background(self, dirs, clamp: bool):
        dirs = np.ascontiguousarray(dirs, np.float64)
        out = np.zeros((len(dirs), 3))
        self.lib.refh_background(self.h, _ptr(dirs), len(dirs), int(clamp), _ptr(out))
        return out

    def photons(self):
        n = self.lib.refh_photon_count(self.h)
        pos = np.zeros((n, 3))
        pw = np.zeros((n, 3))
        leaf = np.zeros(n, np.int32)
        if n:
            self.lib.refh_photons(self.h, _ptr(pos), _ptr(pw), _ptr(leaf))
        return pos, pw, leaf.astype(bool)

    def caustic_query(self, pts, k=15):
        pts = np.ascontiguousarray(pts, np.float64)
        out = np.zeros((len(pts), 3))
        self.lib.refh_caustic_query(self.h, _ptr(pts), len(pts), k, _ptr(out))
        return out


def canonical_scene(scene, ref: "RefOracle | None" = None):
    """Return `scene` with mesh vertices replaced by the positions the reference
    intersects after init_bvh (ft_update_obj_position re-applies a +-1 rad
    rotation in float precision, obj_parser_utils.c:26-46). The CUDA library is
    given these, while both oracles are given the original scene and apply the
    re-transform themselves. Meshes become non-indexed (3 vertices per
    triangle). Uses the reference if given, else the restatement."""
    import copy
    if not scene.meshes:
        return scene
    if ref is not None:
        tp = ref.triangle_positions()
    else:
        ro = Restatement(scene)
        tp = ro.triangle_positions()
        ro.close()
    out = copy.copy(scene)
    out.meshes = []
    base = 0
    for m in scene.meshes:
        nt = len(m.indices)
        pos = tp[base:base + nt].reshape(-1, 3)
        nrm = m.normals[m.indices.reshape(-1)]
        uvs = None if m.uvs is None else m.uvs[m.indices.reshape(-1)]
        idx = np.arange(3 * nt, dtype=np.uint32).reshape(-1, 3)
        out.meshes.append(type(m)(pos, nrm, idx, m.tri_material, uvs, m.material, m.color))
        base += nt
    out._keep = []
    return out


# ------------------------------------------------------------ restatement

RO_HIT_DTYPE = np.dtype([("prim", "<i4"), ("front_face", "<i4"), ("depth", "<i4"),
                         ("material", "<i4"), ("t", "<f8"), ("u", "<f8"), ("v", "<f8"),
                         ("point", "<f8", 3), ("normal", "<f8", 3), ("color", "<f8", 3)])

COUNTER_FIELDS = ["paths", "segments", "shadow_rays", "node_visits", "prim_tests",
                  "sphere_tests", "tri_tests", "plane_tests", "hits", "env_nee",
                  "caustic_gathers"]


class Counters(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in COUNTER_FIELDS]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k in COUNTER_FIELDS}


_rst = None


def rst_lib():
    global _rst
    if _rst is None:
        if not RST_LIB.exists():
            raise FileNotFoundError(f"{RST_LIB} not built (make -C oracle restatement)")
        lib = C.CDLL(str(RST_LIB))
        sig = {
            "ro_create": (_P, [_P]), "ro_destroy": (None, [_P]),
            "ro_set_reference_rng": (None, [C.c_uint64]),
            "ro_get_reference_rng": (C.c_uint64, []),
            "ro_first_hit": (C.c_int, [_P, _P, C.c_int64, _P]),
            "ro_render_reference": (C.c_int, [_P, C.c_int, _P]),
            "ro_render_counter": (C.c_int, [_P, C.c_uint64, C.c_int, C.c_int, C.c_int, _P,
                                            C.c_int64, _P, _P]),
            "ro_trace_path_counter": (C.c_int, [_P, C.c_uint64, C.c_int32, C.c_int32, C.c_int,
                                                _P]),
            "ro_env_tables": (C.c_int, [_P, _P, _P, _P, _P]),
            "ro_env_outcome_probs": (C.c_int64, [_P, _P, _P]),
            "ro_photon_count": (C.c_int64, [_P]),
            "ro_photons": (C.c_int, [_P, _P, _P, _P]),
            "ro_caustic_query": (C.c_int, [_P, _P, C.c_int64, C.c_int, _P]),
            "ro_counters_read": (C.c_int, [_P, _P]),
            "ro_trace_path_events": (C.c_int, [_P, C.c_uint64, C.c_int32, C.c_int32, C.c_int, _P, _P]),
            "ro_path_seed": (C.c_uint64, [C.c_uint64, C.c_uint32, C.c_uint32]),
            "ro_pcg_float": (C.c_float, [C.POINTER(C.c_uint64)]),
            "ro_set_mesh_transform": (None, [C.c_int]),
            "ro_triangle_positions": (C.c_int, [_P, _P]),
            "ro_counters_read": (C.c_int, [_P, _P]),
            "ro_param_count": (C.c_int64, [_P]),
            "ro_set_params": (C.c_int, [_P, _P, C.c_int64, C.c_int]),
        }
        for k, (r, a) in sig.items():
            f = getattr(lib, k)
            f.restype, f.argtypes = r, a
        _rst = lib
    return _rst


class Restatement:
    """This project's FP64 restatement of the reference path (oracle/mrt_oracle.c)."""

    def __init__(self, scene):
        self.lib = rst_lib()
        self.scene = scene
        self.desc = scene.desc()
        self.h = self.lib.ro_create(C.byref(self.desc))
        if not self.h:
            raise ValueError("ro_create rejected the scene")
        self.W, self.H = scene.width, scene.height

    def close(self):
        if self.h:
            self.lib.ro_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def set_seed(seed: int):
        rst_lib().ro_set_reference_rng(seed)

    def first_hit(self, orig, dirs):
        rays = np.ascontiguousarray(np.concatenate([orig, dirs], 1), np.float64)
        out = np.zeros(len(rays), RO_HIT_DTYPE)
        self.lib.ro_first_hit(self.h, _ptr(rays), len(rays), _ptr(out))
        return out

    def render_reference(self, spp: int) -> np.ndarray:
        acc = np.zeros((self.H, self.W, 3))
        self.lib.ro_render_reference(self.h, spp, _ptr(acc))
        return acc

    def render_counter(self, seed: int, spp: int, sample_base: int = 0, jitter: int = 0,
                       pix: np.ndarray | None = None):
        if pix is None:
            acc = np.zeros((self.H * self.W, 3))
            n = 0
        else:
            pix = np.ascontiguousarray(pix, np.int32)
            acc = np.zeros((len(pix), 3))
            n = len(pix)
        cnt = Counters()
        self.lib.ro_render_counter(self.h, seed, sample_base, spp, jitter, _ptr(pix), n,
                                   _ptr(acc), C.byref(cnt))
        return acc, cnt.as_dict()

    def path(self, seed: int, pixel: int, sample: int, jitter: int = 0):
        out = np.zeros(3)
        self.lib.ro_trace_path_counter(self.h, seed, pixel, sample, jitter, _ptr(out))
        return out

    def path_events(self, seed: int, pixel: int, sample: int, jitter: int = 0):
        ev = np.zeros((16, 20))
        rgb = np.zeros(3)
        self.lib.ro_trace_path_events(self.h, seed, pixel, sample, jitter, _ptr(ev), _ptr(rgb))
        return ev, rgb

    def env_tables(self):
        if self.scene.hdr is None:
            return None
        h, w = self.scene.hdr.shape[:2]
        pdf = np.zeros(w * h, np.float32)
        cm = np.zeros(h, np.float32)
        cc = np.zeros(w * h, np.float32)
        avg = C.c_double(0)
        self.lib.ro_env_tables(self.h, _ptr(pdf), _ptr(cm), _ptr(cc), C.byref(avg))
        return pdf, cm, cc, avg.value

    def env_outcome_probs(self):
        h, w = self.scene.hdr.shape[:2]
        n = (h - 1) * (w + 1)
        p = np.zeros(n)
        j = np.zeros(n, np.int32)
        k = self.lib.ro_env_outcome_probs(self.h, _ptr(p), _ptr(j))
        return p[:k], j[:k]

    def triangle_positions(self):
        out = np.zeros((self.scene.n_triangles, 9))
        self.lib.ro_triangle_positions(self.h, _ptr(out))
        return out

    def photons(self):
        n = self.lib.ro_photon_count(self.h)
        pos = np.zeros((n, 3))
        pw = np.zeros((n, 3))
        leaf = np.zeros(n, np.int32)
        if n:
            self.lib.ro_photons(self.h, _ptr(pos), _ptr(pw), _ptr(leaf))
        return pos, pw, leaf.astype(bool)

    def caustic_query(self, pts, k=15):
        pts = np.ascontiguousarray(pts, np.float64)
        out = np.zeros((len(pts), 3))
        self.lib.ro_caustic_query(self.h, _ptr(pts), len(pts), k, _ptr(out))
        return out

    def param_count(self) -> int:
        return int(self.lib.ro_param_count(self.h))

    def set_params(self, theta, exact: bool = True) -> None:
        """Differentiable parameters in mrt_forward's layout (albedo, roughness,
        emission, linear sky); exact keeps every intermediate in double."""
        theta = np.ascontiguousarray(theta, np.float64)
        if self.lib.ro_set_params(self.h, _ptr(theta), len(theta), int(exact)) != 0:
            raise ValueError(f"theta has {len(theta)} entries, the scene {self.param_count()}")

    def linear_functional(self, theta, weights, seed: int, spp: int, pix, sample_base: int = 0,
                          jitter: int = 0, exact: bool = True) -> float:
        """sum(weights * mean-over-spp radiance) over the pixels `pix`
        (counter RNG, the GPU's paths)."""
        self.set_params(theta, exact)
        acc, _ = self.render_counter(seed, spp, sample_base, jitter, pix)
        return float(np.sum(np.asarray(weights, np.float64) * acc / spp))

    def fd_gradient(self, theta, directions, weights, seed: int, spp: int, pix, h: float = 1e-6,
                    sample_base: int = 0, jitter: int = 0) -> np.ndarray:
        """FP64 reference gradient of linear_functional along each direction
        (rows of `directions`): central differences with common random
        numbers in exact mode, step h."""
        theta = np.asarray(theta, np.float64)
        out = []
        for v in np.atleast_2d(directions):
            fp = self.linear_functional(theta + h * v, weights, seed, spp, pix, sample_base, jitter)
            fm = self.linear_functional(theta - h * v, weights, seed, spp, pix, sample_base, jitter)
            out.append((fp - fm) / (2 * h))
        self.set_params(theta, True)
        return np.array(out)


def pcg_stream(seed: int, pixel: int, sample: int, n: int) -> np.ndarray:
    """First n floats of the counter-based stream of (seed, pixel, sample)."""
    lib = rst_lib()
    st = C.c_uint64(lib.ro_path_seed(seed, pixel, sample))
    return np.array([lib.ro_pcg_float(C.byref(st)) for _ in range(n)], np.float32)
