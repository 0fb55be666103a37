"""Generates the converged-radiance fixtures (conv_<config>.npz) from the
reference itself. TEST INFRASTRUCTURE: run here, where the reference is
compiled from its sources into oracle/_ref/liboracle_ref.so.

For each benchmark configuration the reference's own CPU path renders a set
of pixels at 4096 samples per pixel: calc_one_sample_task
(src/ray_tracing/calc_sample.c:44) on each listed pixel, one shared
vec3_random() offset per sample as calc_one_sample (calc_sample.c:73) draws
it, through the harness call refh_render_pixels. Pixels:
  c0  every pixel of the 320x240 frame;
  c1, c2, c4  a seeded stratified subset of 4,096 pixels (one uniformly drawn
      pixel in each cell of a 64x64 grid over the frame).
The samples are split into B batches rendered by forked processes, each with
its own seed of the reference's global xorshift (random.c:27), so that every
fixture stores, per pixel, the mean and the variance of the mean estimated
from the B batch means, and, per batch, the mean over the listed pixels
(the image-mean bias test needs it: pixels of one batch share offsets).

c2 runs in the reference's single-pass kNN mode (k = 15, 2 M photons). The
photon map is the one the reference builds for RNG seed PHOTON_SEED; the
fixture stores a digest of its leaf photons, and the GPU test rebuilds the
same map with the compiled reference and uploads it, because a kNN image
depends on its photon set and that noise does not average out over samples.

  python tests/golden/make_converged.py [c0 c1 c2 c4] [--procs N]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO / "42-minirt_b200"))
sys.path.insert(0, str(REPO / "oracle"))

SPP = 4096
BATCHES = 64
PHOTON_SEED = 12345
SUBSET = 64          # SUBSET x SUBSET strata -> 4,096 pixels


def make_scene(name: str):
    import scenes
    return {"c0": scenes.make_c0, "c1": scenes.make_c1, "c2": scenes.make_c2, "c4": scenes.make_c4}[name]()


def stratified_pixels(width: int, height: int, seed: int, n: int = SUBSET) -> np.ndarray:
    """One uniformly drawn pixel per cell of an n x n grid over the frame,
    as linear indices y * width + x (row-major, the reference's pixel index)."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0, width, n + 1).astype(np.int64)
    ys = np.linspace(0, height, n + 1).astype(np.int64)
    out = []
    for j in range(n):
        for i in range(n):
            x = rng.integers(xs[i], max(xs[i + 1], xs[i] + 1))
            y = rng.integers(ys[j], max(ys[j + 1], ys[j] + 1))
            out.append(y * width + x)
    return np.array(out, np.int32)


def pixel_set(name: str, sc) -> np.ndarray:
    if name == "c0":
        return np.arange(sc.width * sc.height, dtype=np.int32)
    return stratified_pixels(sc.width, sc.height, seed=1000 + sc.seed)


def photon_digest(pos: np.ndarray, power: np.ndarray) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(pos, np.float64).tobytes())
    h.update(np.ascontiguousarray(power, np.float64).tobytes())
    return h.hexdigest()


def batch_seed(name: str, b: int) -> int:
    return 0x9E3779B97F4A7C15 ^ (hash_name(name) * 1000003 + 7919 * (b + 1))


def hash_name(name: str) -> int:
    return int.from_bytes(hashlib.sha256(name.encode()).digest()[:4], "little")


def _worker(ref, name: str, pix: np.ndarray, batches: list[int], spp_b: int, out_dir: str) -> None:
    W = ref.W
    py, px = pix // W, pix % W
    for b in batches:
        ref.set_seed(batch_seed(name, b) & 0xFFFFFFFFFFFFFFFF or 1)
        ref.clear()
        ref.render_pixels(pix, spp_b)
        acc = ref.accum()[py, px] / spp_b
        np.save(os.path.join(out_dir, f"b{b:04d}.npy"), acc)


def render(name: str, procs: int, spp: int = SPP, batches: int = BATCHES) -> dict:
    import oracle
    sc = make_scene(name)
    t0 = time.perf_counter()
    oracle.ref_lib().refh_set_seed(PHOTON_SEED)
    ref = oracle.RefOracle(sc)
    prep = time.perf_counter() - t0
    pix = pixel_set(name, sc)
    spp_b = spp // batches
    extra = {}
    if sc.caustic is not None:
        pos, pw, leaf = ref.photons()
        extra["photon_digest"] = photon_digest(pos[leaf], pw[leaf])
        extra["photons_in_leaf"] = int(leaf.sum())
    t1 = time.perf_counter()
    with tempfile.TemporaryDirectory() as tmp:
        pids = []
        for p in range(procs):
            pid = os.fork()
            if pid == 0:
                code = 0
                try:
                    _worker(ref, name, pix, list(range(p, batches, procs)), spp_b, tmp)
                except BaseException:  # noqa: BLE001 - report through the exit code
                    code = 1
                os._exit(code)
            pids.append(pid)
        for pid in pids:
            _, status = os.waitpid(pid, 0)
            if status != 0:
                raise RuntimeError(f"{name}: a render worker failed")
        bm = np.stack([np.load(os.path.join(tmp, f"b{b:04d}.npy")) for b in range(batches)])
    secs = time.perf_counter() - t1
    ref.close()
    mean = bm.mean(0)
    var_mean = bm.var(0, ddof=1) / batches
    return dict(config=name, pixels=pix, mean=mean.astype(np.float32), var_mean=var_mean.astype(np.float32),
                batch_image_mean=bm.mean(1), spp=spp, batches=batches, width=sc.width, height=sc.height,
                depth=sc.max_bounces, prep_seconds=prep, render_seconds=secs, procs=procs, **extra)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("configs", nargs="*", default=["c0", "c1", "c2", "c4"])
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--spp", type=int, default=SPP)
    a = ap.parse_args()
    for name in a.configs:
        r = render(name, a.procs, a.spp)
        meta = {k: v for k, v in r.items() if not isinstance(v, np.ndarray)}
        arrays = {k: v for k, v in r.items() if isinstance(v, np.ndarray)}
        np.savez_compressed(HERE / f"conv_{name}.npz", meta=json.dumps(meta), **arrays)
        print(json.dumps(meta), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
