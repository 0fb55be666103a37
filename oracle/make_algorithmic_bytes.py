"""MEASUREMENT INFRASTRUCTURE — canonical algorithmic bytes per path.

The roofline's `achieved` figure divides a fixed, implementation-independent
byte count per path by the measured kernel time. That count comes from the
oracle restatement: it traces a seeded sample of camera paths of each
workload through the reference's own median-split BVH topology
(bvh_build.c:16-127) with a closest-hit, near-first, t-culled traversal,
and prices every access with the per-unit sizes below:
  32 B per BVH node, 48 B per triangle test, 16 B per sphere test,
  48 B per cylinder / cone / hyperboloid test, 32 B per plane test, 80 B per traced ray (32 read + 32 write + 16 hit
  record), 160 B per shading event (64 vertex normals/uv + 96 material
  record), 28 B per HDRI importance sample (8 inverse tables + 4 pdf + 16
  texel), plus 12 B / spp for the frame buffer. Texel fetches of textured
  scenes are not priced (so t0's figure is a lower bound).
The result is frozen in oracle/algorithmic_bytes.json so kernel or BVH
changes cannot move it.  Run:  python oracle/make_algorithmic_bytes.py [config ...]
(named configs only: the other entries of the file are kept as they are).
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent / "42-minirt_b200"))
sys.path.insert(0, str(HERE))
import oracle  # noqa: E402
import scenes  # noqa: E402

UNIT = dict(node=32, tri=48, sphere=16, quadric=48, plane=32, ray=80, hit=160, env=28, fb=12)


def bytes_per_path(cnt: dict, spp: int) -> float:
    p = max(cnt["paths"], 1)
    quadric_tests = cnt["prim_tests"] - cnt["sphere_tests"] - cnt["tri_tests"]
    b = (UNIT["node"] * cnt["node_visits"] + UNIT["tri"] * cnt["tri_tests"]
         + UNIT["sphere"] * cnt["sphere_tests"] + UNIT["quadric"] * quadric_tests
         + UNIT["plane"] * cnt["plane_tests"]
         + UNIT["ray"] * (cnt["segments"] + cnt["shadow_rays"]) + UNIT["hit"] * cnt["hits"]
         + UNIT["env"] * cnt["env_nee"])
    return b / p + UNIT["fb"] / spp


def main(only=None):
    path = HERE / "algorithmic_bytes.json"
    out = json.loads(path.read_text()) if only and path.exists() else {"configs": {}}
    out["units"] = UNIT
    cases = [("c0", scenes.make_c0, 64, 20000), ("c1", scenes.make_c1, 256, 4000),
             ("c2", lambda: scenes.make_c2(photons=20000), 128, 4000),
             ("c4", scenes.make_c4, 64, 4000), ("q0", scenes.make_quadrics, 64, 20000),
             ("t0", scenes.make_textured, 64, 20000)]
    for name, make, spp, n in cases:
        if only and name not in only:
            continue
        sc = make()
        t = time.time()
        ro = oracle.Restatement(sc)
        prep = time.time() - t
        rng = np.random.default_rng(7)
        pix = rng.integers(0, sc.width * sc.height, n).astype(np.int32)
        _, cnt = ro.render_counter(3, 1, pix=pix)
        bpp = bytes_per_path(cnt, spp)
        out["configs"][name] = {"bytes_per_path": bpp, "counters": cnt, "sample_paths": n,
                                "spp": spp, "prep_seconds": prep}
        print(name, round(bpp, 1), cnt, flush=True)
        ro.close()
    path.write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main(sys.argv[1:])
