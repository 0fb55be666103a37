"""TEST/MEASUREMENT INFRASTRUCTURE — times the reference's own CPU path.

The reference renders on one thread with one global RNG
(src/ray_tracing/calc_sample.c:96-97, src/math/random.c:27), so the
multi-core CPU baseline is P forked processes, each with its own RNG state,
rendering random pixel batches through calc_one_sample_task
(calc_sample.c:44) of the reference compiled from its sources
(oracle/_ref/liboracle_ref.so). Scene preparation (the reference's BVH build,
HDRI tables, photon map) happens once before forking and is not timed.

Two builds of the same sources (oracle/Makefile): "parity" (-O2, the build
the parity tests pin against) and "fast" (-O3 -march=x86-64-v3, no
-ffast-math), the stronger of the two CPU baselines.

Run as a separate process (it forks; it must not share a process with CUDA):
  python oracle/cpu_baseline.py --config c1 --seconds 10 [--procs N] [--steps K --warmup W]
                                [--build parity|fast]
Prints one JSON object.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent / "42-minirt_b200"))
sys.path.insert(0, str(HERE))


def make_scene(config: str):
    import scenes
    return scenes.CONFIGS[config]()


def _worker(h_ref, seed: int, seconds: float, npix: int, batch: int, wfd: int) -> None:
    import oracle
    lib = oracle.ref_lib()
    lib.refh_set_seed(seed)
    rng = np.random.default_rng(seed)
    paths = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        pix = rng.integers(0, npix, batch).astype(np.int32)
        lib.refh_render_pixels(h_ref, pix.ctypes.data, batch, 1)
        paths += batch
    dt = time.perf_counter() - t0
    os.write(wfd, json.dumps({"paths": paths, "seconds": dt}).encode())
    os.close(wfd)


def timed_step(ref, seconds: float, procs: int, seed: int, batch: int) -> dict:
    """One bounded sample: `procs` forked workers render for `seconds`."""
    npix = ref.W * ref.H
    pipes, pids = [], []
    for p in range(procs):
        r, w = os.pipe()
        pid = os.fork()
        if pid == 0:
            os.close(r)
            try:
                _worker(ref.h, seed * 1009 + p * 7919 + 1, seconds, npix, batch, w)
            finally:
                os._exit(0)
        os.close(w)
        pipes.append(r)
        pids.append(pid)
    res = []
    for r in pipes:
        data = b""
        while True:
            chunk = os.read(r, 4096)
            if not chunk:
                break
            data += chunk
        os.close(r)
        res.append(json.loads(data.decode()))
    for pid in pids:
        os.waitpid(pid, 0)
    paths = sum(x["paths"] for x in res)
    secs = max(x["seconds"] for x in res)
    return {"paths": paths, "seconds": secs, "mpaths_s": paths / secs / 1e6}


BUILDS = {"parity": ("_ref/liboracle_ref.so", "-O2"),
          "fast": ("_ref/fast/liboracle_ref.so", "-O3 -march=x86-64-v3")}


def run(config: str, seconds: float, procs: int, steps: int = 1, warmup: int = 0,
        batch: int = 64, build: str = "parity") -> dict:
    import oracle
    oracle.REF_LIB = HERE / BUILDS[build][0]
    sc = make_scene(config)
    t0 = time.perf_counter()
    oracle.ref_lib().refh_set_seed(12345)
    ref = oracle.RefOracle(sc)
    prep = time.perf_counter() - t0
    for w in range(warmup):
        timed_step(ref, min(seconds, 2.0), procs, 1000 + w, batch)
    rates = [timed_step(ref, seconds, procs, s + 1, batch) for s in range(steps)]
    paths = sum(r["paths"] for r in rates)
    secs = sum(r["seconds"] for r in rates)
    return {"config": config, "procs": procs, "prep_seconds": prep, "paths": paths,
            "seconds": secs, "mpaths_s": paths / secs / 1e6,
            "per_core_mpaths_s": paths / secs / 1e6 / procs, "steps": steps,
            "step_mpaths_s": [r["mpaths_s"] for r in rates],
            "build": f"{build} ({BUILDS[build][1]}, no -ffast-math)",
            "sample": f"{config} full scene, random pixels in batches of {batch} at 1 spp, "
                      f"{procs} forked processes x {seconds:g} s per step"}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c1")
    ap.add_argument("--seconds", type=float, default=10.0)
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=0)
    ap.add_argument("--build", default="parity", choices=sorted(BUILDS))
    a = ap.parse_args()
    print(json.dumps(run(a.config, a.seconds, a.procs, a.steps, a.warmup, build=a.build)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
