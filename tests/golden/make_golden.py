"""Generates the golden fixtures in this folder from the reference itself.

The reference (miniRT) ships no tests or golden vectors, so the fixtures are
outputs of its own CPU code, compiled from its sources by oracle/Makefile into
oracle/_ref/liboracle_ref.so, on small seeded scenes:
  * first-hit records of hit_register_all on seeded rays,
  * float_render after N samples of calc_one_sample with a fixed RNG state,
  * HDRI tables of make_importance_sampling_map,
  * the photon map of caustic_manager and kNN caustic estimates.
Run here (where the reference is mounted):  python tests/golden/make_golden.py [case ...]
The GPU box has no reference; tests there read these files.
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO / "42-minirt_b200"))
sys.path.insert(0, str(REPO / "oracle"))
import oracle  # noqa: E402
import scenes  # noqa: E402

CASES = {
    "c0": dict(make=lambda: scenes.make_c0(0, 32, 24, depth=8), spp=4),
    "c1": dict(make=lambda: scenes.make_c1(1, 24, 16, depth=6, freq=12, sky=(48, 24)), spp=2),
    "c2": dict(make=lambda: scenes.make_c2(2, 24, 16, depth=6, grid=16, photons=3000), spp=2),
    "q0": dict(make=lambda: scenes.make_quadrics(5, 32, 24, depth=6), spp=4),
    "t0": dict(make=lambda: scenes.make_textured(6, 32, 24, depth=6), spp=4),
}


def scene_digest(sc) -> str:
    h = hashlib.sha256()
    for m in sc.materials:
        h.update(repr(sorted(m.items())).encode())
    for s in sc.spheres:
        h.update(repr(s).encode())
    for p in sc.planes:
        h.update(repr(p).encode())
    for q in sc.cylinders + sc.cones + sc.hyperboloids:
        h.update(repr(sorted(q.items())).encode())
    for t in sc.textures:
        h.update(repr(sorted((k, v) for k, v in t.items() if k != "rgba")).encode())
        if t.get("rgba") is not None:
            h.update(np.ascontiguousarray(t["rgba"]).tobytes())
    for m in sc.meshes:
        for a in (m.positions, m.normals, m.indices, m.tri_material):
            if a is not None:
                h.update(np.ascontiguousarray(a).tobytes())
    if sc.hdr is not None:
        h.update(sc.hdr.tobytes())
    h.update(repr(sc.camera).encode())
    return h.hexdigest()


def rays_for(ref, n=4096, seed=0):
    vp = ref.viewport()
    rng = np.random.default_rng(seed)
    o = vp["cam"][None] + rng.normal(size=(n, 3)) * 0.3
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    # half of them camera rays through random pixels (unnormalised, like calc_one_sample_task)
    k = n // 2
    px = rng.uniform(0, ref.W, k)
    py = rng.uniform(0, ref.H, k)
    o[:k] = vp["cam"]
    d[:k] = vp["pixel00"][None] + vp["du"][None] * px[:, None] + vp["dv"][None] * py[:, None] - vp["cam"][None]
    return o, d


def main(names=None):
    for name, case in CASES.items():
        if names and name not in names:
            continue
        sc = case["make"]()
        oracle.ref_lib().refh_set_seed(4242)
        ref = oracle.RefOracle(sc)
        out = {"digest": np.array(scene_digest(sc))}
        o, d = rays_for(ref)
        hits = ref.first_hit(o, d)
        out.update(rays_o=o, rays_d=d)
        for f in ("prim", "front_face", "depth", "t", "u", "v", "point", "normal", "color"):
            out["hit_" + f] = hits[f]
        ref.set_seed(777)
        offs = ref.render(case["spp"])
        out.update(render=ref.accum(), render_offsets=offs, render_seed=np.array(777),
                   render_spp=np.array(case["spp"]))
        et = ref.env_tables()
        if et is not None:
            out.update(pdf_joint=et[0], cdf_m_inv=et[1], cdf_c_inv=et[2], column_average=np.array(et[3]))
        pos, pw, leaf = ref.photons()
        if len(pos):
            rng = np.random.default_rng(5)
            q = pos[rng.integers(0, len(pos), 256)] + rng.normal(size=(256, 3)) * 0.02
            out.update(photon_pos=pos, photon_pow=pw, photon_in_leaf=leaf, caustic_q=q,
                       caustic_rgb=ref.caustic_query(q, 15))
        if sc.meshes:
            out["tri_positions"] = ref.triangle_positions()
        ref.close()
        np.savez_compressed(HERE / f"{name}_pins.npz", **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main(sys.argv[1:])
