"""Benchmark of the path-tracing hot path (one JSON line on rank 0).

Metric: Mpaths/s (camera paths through the reference's estimator per second,
whole job) on the 1920x1080 / 256 spp / depth 12 workload: a 1,310,720
triangle displaced geodesic sphere with 16 materials under a 2048x1024 RGBE
sky sampled by importance (seeded synthetic scene; the reference publishes no
benchmark scene). One step = one pass over the frame at --spp-per-step
samples per pixel (16 steps = the 256 spp render).

  value       device time (CUDA events on the library's stream) of the timed
              steps, inputs resident in HBM; the best of the forms (plain
              one-path-per-thread megakernel, persistent regenerating
              megakernel, wavefront), each reported under "forms".
  relmse      time to relMSE <= 1e-3 against the reference's own CPU render
              at 4096 spp (tests/golden/conv_<config>.npz, a stratified
              subset of 4,096 pixels): the best form renders progressively
              until relMSE against the converged image (reference noise
              subtracted) is <= 1e-3; measured device time to that point,
              and that sample count at each other form's rate.
  e2e         the same render through the C-ABI a reference host calls:
              per step a camera upload, the render and a device->host read of
              the frame accumulated into a pinned double buffer
              (t_fcolor float_render), wall-clocked.
  roofline    canonical algorithmic bytes per path (oracle/algorithmic_bytes.json,
              reference BVH topology) x paths per launch / mean launch time,
              against the measured HBM copy bandwidth.
  cpu_baseline the reference's own CPU code (compiled from its sources) on
              this host's cores, timed in a separate process.
  adjoint     the differentiable workload (512x512, 64 spp, depth 8,
              200,000-triangle sphere, 32 materials, 512x256 sky):
              device time of mrt_forward and mrt_backward (path-replay
              adjoint) and their ratio, then 100 projected Adam steps
              (lr 1e-2 on a cosine schedule, sky texels in log space, a
              128-spp residual and a decorrelated 64-spp gradient per step)
              from the scene's parameters towards a 1024-spp target rendered
              at parameters perturbed by +-20%, for three seeds (median
              reported), with the material error over all material entries
              and over those the image depends on.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun each rank renders its own sample range (weak scaling); the
frames are summed on rank 0 by the library's mrt_reduce_frame (NCCL) inside
the timed regions: once after the timed steps of each form, and after every
step of the end-to-end run.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "42-minirt_b200"))

METRIC = "Mpaths/s and time to relMSE<=1e-3, wavefront vs plain megakernel, 1 B200"
UNIT = "Mpaths/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1")
    ap.add_argument("--spp-per-step", type=int, default=16)
    ap.add_argument("--forms", default="megakernel_plain,megakernel,wavefront")
    ap.add_argument("--no-relmse", action="store_true")
    ap.add_argument("--relmse-cap-spp", type=int, default=None,
                    help="most samples per pixel rendered while waiting for relMSE <= 1e-3 "
                         "(default: 16384 for c0, whose emitter-lit frame converges slowly "
                         "but renders in a fraction of a second, else 4096)")
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--adam-steps", type=int, default=100)
    ap.add_argument("--only-adjoint", action="store_true",
                    help="run only the differentiable workload and print its figures (profiling aid)")
    ap.add_argument("--adjoint-res", type=int, default=512)
    return ap.parse_args()


class Clocks:
    """nvidia-smi sampling during the timed region (clocks and throttle reasons)."""

    def __init__(self, index: int):
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        rows = [r.split(", ") for r in self.path.read_text().strip().splitlines() if r.strip()]
        self.path.unlink(missing_ok=True)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for k, name in enumerate(names):
                if r[5 + k].strip() == "Active":
                    reasons.add(name)
        loaded = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(rows)}


def cpu_baseline(config: str, seconds: float, steps: int = 1, warmup: int = 0,
                 build: str = "fast") -> dict | None:
    """The reference's CPU path, in a fresh process (it forks workers).
    build: "fast" (-O3 -march=x86-64-v3, no -ffast-math; the stronger
    baseline, reported as the value) or "parity" (-O2, the build the parity
    tests pin against)."""
    script = REPO / "oracle" / "cpu_baseline.py"
    lib = REPO / "oracle" / "_ref" / ("fast/liboracle_ref.so" if build == "fast" else "liboracle_ref.so")
    if not lib.exists():
        return None
    out = subprocess.run([sys.executable, str(script), "--config", config, "--seconds", str(seconds),
                          "--steps", str(steps), "--warmup", str(warmup), "--build", build],
                         capture_output=True, text=True, timeout=1800)
    for line in out.stdout.splitlines()[::-1]:
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError("cpu baseline failed: " + out.stderr[-2000:])


def run_reference_arm(a) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # both builds of the reference on all host cores; the faster one is the
    # arm's value, the other is reported beside it
    runs = [x for x in (cpu_baseline(a.config, a.cpu_seconds, steps=a.steps, warmup=a.warmup, build=b)
                        for b in ("fast", "parity")) if x is not None]
    r = max(runs, key=lambda x: x["mpaths_s"]) if runs else None
    rp = ([x for x in runs if x is not r] or [None])[0]
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/liboracle_ref.so (the reference compiled from its "
                          "sources) is not present"}))
        return
    line = {"impl": "reference", "metric": METRIC, "value": r["mpaths_s"], "unit": UNIT,
            "n_gpus": 0, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1000.0 * r["seconds"] / max(a.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(a, None),
            "cpu_baseline": {"value": r["mpaths_s"], "unit": UNIT, "cores": r["procs"],
                             "kind": "reference", "sample": r["sample"], "build": r["build"],
                             "other_build": None if rp is None else
                             {"value": rp["mpaths_s"], "build": rp["build"]}},
            "e2e": {"value": r["mpaths_s"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def convergence(ctx, sc, config: str, spp_step: int, forms: dict, fid: int, cap_spp: int) -> dict:
    """Time to relMSE <= 1e-3 against the reference CPU render at 4096 spp.

    The comparator is the converged-radiance fixture tests/golden/conv_<config>.npz:
    the reference's own calc_one_sample_task at 4096 samples per pixel on a
    seeded stratified subset of 4,096 pixels (every pixel for c0), with the
    variance of each pixel's mean. The best form renders the frame
    progressively (spp_step samples per call); after each call its image is
    compared at the fixture's pixels with relMSE against the converged image,
    mean(((x - r)^2 - var_r) / (r^2 + 0.01)) (the reference's own noise
    var_r subtracted). The time is the device time of the calls up to the
    first one at or below 1e-3, rendered, not extrapolated; for the other
    forms (same estimator, same paths) it is that sample count at their
    measured rate. c = relMSE * N fitted over the run is reported beside it."""
    import convergence as cv
    import mrt
    path = REPO / "tests" / "golden" / f"conv_{config}.npz"
    if not path.exists():
        return {"unavailable": f"no converged-radiance fixture for {config}"}
    fx = cv.load_fixture(path)
    pix, r, var_r = fx["pixels"], fx["mean"].astype(np.float64), fx["var_mean"].astype(np.float64)
    ctx.clear()
    done, ms, trace, reached = 0, 0.0, [], None
    while done < cap_spp:
        st = ctx.render(spp_step, seed=31, sample_base=done, form=fid,
                        use_graph=1 if fid == mrt.FORM_WAVEFRONT else 0)
        ms += st.ms
        done += spp_step
        img, n = ctx.read_accum()
        x = cv.pixel_values(img / n, pix)
        rc = cv.relmse_converged(x, r, var_r)
        trace.append((done, rc))
        if rc <= 1e-3:
            reached = (done, ms, rc, cv.relmse(x, r))
            break
    ctx.clear()
    ns = np.array([t[0] for t in trace], np.float64)
    rs = np.array([t[1] for t in trace], np.float64)
    keep = ns >= 4 * spp_step
    c = float(np.sum(rs[keep] / ns[keep]) / np.sum(1.0 / ns[keep] ** 2)) if keep.any() else None
    npix = sc.width * sc.height
    out = {"ref": "reference CPU render, 4096 spp (tests/golden/conv_%s.npz, %d pixels)" % (config, len(pix)),
           "relmse_definition": "mean(((x-r)^2 - var_r)/(r^2+0.01)) at the fixture's pixels: "
                                "relMSE against the converged image the reference estimates",
           "relmse_ref_noise": float(np.mean(var_r / (r ** 2 + 1e-2))),
           "c_fit": c, "trace": [[int(a), float(b)] for a, b in trace[:: max(1, len(trace) // 16)]]}
    if config.startswith("c2"):
        out["note"] = ("a kNN caustic image depends on its photon set: this render gathers the "
                       "library's own photon map, the fixture the reference's, so relMSE levels "
                       "off at their difference; the converged-radiance test gives the GPU the "
                       "reference's photon map (mrt_set_photons) and meets the bar")
    if reached is None:
        out.update({"reached": False, "spp_rendered": done, "relmse_last": float(rs[-1])})
        return out
    spp_hit, ms_hit, rc_hit, raw_hit = reached
    out.update({"reached": True, "spp_to_1e-3": spp_hit, "relmse_at_stop": rc_hit,
                "relmse_raw_at_stop": raw_hit, "measured_form_ms": ms_hit})
    for name, f in forms.items():
        if "value" in f:
            out[f"time_to_1e-3_s_{name}"] = (ms_hit / 1000.0 if form_ids_name(fid) == name
                                             else spp_hit * npix / (f["value"] * 1e6))
    return out


def form_ids_name(fid: int) -> str:
    import mrt
    return {mrt.FORM_MEGAKERNEL: "megakernel", mrt.FORM_WAVEFRONT: "wavefront",
            mrt.FORM_MEGAKERNEL_PLAIN: "megakernel_plain"}.get(fid, "?")


def adjoint_bench(device: int, adam_steps: int, res: int = 512) -> dict:
    """Forward / backward cost and an Adam fit on the differentiable workload."""
    import mrt
    import scenes
    sc = scenes.make_c4(width=res, height=res)
    ctx = mrt.Context(sc.width, sc.height, device=device)
    ctx.build(sc)
    th = ctx.diff_params()
    spp = 64
    w = np.random.default_rng(0).uniform(0.5, 1.5, (sc.height, sc.width, 3)).astype(np.float32)
    fwd, bwd = [], []
    for i in range(4):
        _, sf = ctx.forward(th, spp=spp, seed=1 + i, stats=True)
        _, sb = ctx.backward(th, w, spp=spp, seed=1 + i, stats=True)
        if i:                                   # the first pair is warm-up
            fwd.append(sf.ms)
            bwd.append(sb.ms)
    paths = sc.width * sc.height * spp
    out = {"workload": f"c4: {res}x{res}, 64 spp, depth 8, 200,000-triangle displaced sphere, "
                       "32 materials, 512x256 RGBE sky",
           "forward_ms": statistics.median(fwd), "backward_ms": statistics.median(bwd),
           "backward_over_forward": statistics.median(bwd) / statistics.median(fwd),
           "forward_mpaths_s": paths / statistics.median(fwd) / 1e3,
           "backward_mpaths_s": paths / statistics.median(bwd) / 1e3}
    if adam_steps > 0:
        try:
            import torch
            import inverse
        except ImportError:
            return out
        lay = ctx.diff_layout()
        target_theta = inverse.perturb(th, lay, 0.2, seed=4)
        target = torch.tensor(ctx.forward(target_theta, spp=1024, seed=4242), device=f"cuda:{device}")
        nm = 5 * (lay["albedo"] // 3)
        # material entries the image depends on: non-zero gradient at the start
        # (roughness of a lambertian material, for one, moves nothing)
        g0 = ctx.backward(th, np.ones((sc.height, sc.width, 3), np.float32), spp=64, seed=7)
        seen = np.nonzero(g0[:nm] != 0)[0]
        runs = []
        for fit_seed in (1000, 2000, 3000):
            t0 = time.perf_counter()
            # the joint fit keeps the sky in log space and the full image
            # gradient: in linear space one of three seeds diverged, and the
            # clip below biased the sun texels' gradients, whose error the
            # albedos then absorbed (material error 0.047-0.050 vs 0.040)
            fit, losses = inverse.fit(ctx, th, target, steps=adam_steps, lr=1e-2, spp=spp, seed=fit_seed,
                                      residual_spp=128, lr_decay=True, sky_log=True)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            fit = fit.cpu().numpy()
            runs.append({"seed": fit_seed, "loss_first": losses[0], "loss_last": float(np.mean(losses[-5:])),
                         "wall_s": wall,
                         "material_param_mae_start": float(np.abs(th[:nm] - target_theta[:nm]).mean()),
                         "material_param_mae_end": float(np.abs(fit[:nm] - target_theta[:nm]).mean()),
                         "seen_param_mae_start": float(np.abs(th[seen] - target_theta[seen]).mean()),
                         "seen_param_mae_end": float(np.abs(fit[seen] - target_theta[seen]).mean())})
        med = sorted(runs, key=lambda r: r["loss_last"])[1]
        # the materials alone, under the target's sky: the joint fit cannot
        # tell a brighter sky from brighter albedos, this one can
        na = lay["albedo"]
        init = target_theta.copy()
        init[:nm] = th[:nm]
        mask = np.zeros_like(th)
        mask[:nm] = 1
        t0 = time.perf_counter()
        fit, losses = inverse.fit(ctx, init, target, steps=adam_steps, lr=1e-2, spp=spp, seed=1000,
                                  residual_spp=128, lr_decay=True, mask=mask, grad_quantile=0.999)
        torch.cuda.synchronize()
        fit = fit.cpu().numpy()
        mat_only = {"loss_first": losses[0], "loss_last": float(np.mean(losses[-5:])),
                    "wall_s": time.perf_counter() - t0,
                    "albedo_mae_start": float(np.abs(init[:na] - target_theta[:na]).mean()),
                    "albedo_mae_end": float(np.abs(fit[:na] - target_theta[:na]).mean()),
                    "seen_param_mae_start": float(np.abs(init[seen] - target_theta[seen]).mean()),
                    "seen_param_mae_end": float(np.abs(fit[seen] - target_theta[seen]).mean())}
        out["adam"] = {"steps": adam_steps, "lr": 1e-2, "spp": spp, "residual_spp": 128,
                       "schedule": "cosine decay to 1% of lr; joint fit: sky texels in log space; "
                                   "materials-only fit: image gradient clipped per pixel at its 99.9th "
                                   "percentile",
                       "seen_material_entries": int(len(seen)), "of_material_entries": nm,
                       "median_of_3_seeds": med, "runs": runs, "materials_only_under_target_sky": mat_only}
    ctx.close()
    return out


def bench_c3(a) -> int:
    """Batched uneven workload: 64 scenes (log-uniform 10k-2M triangles,
    256^2-1024^2 pixels, 16-256 spp, depth 8-16, half HDRI half area light).
    One step renders spp_i / 16 samples of every scene; 16 steps are the whole
    workload. Forms: one persistent launch over all scenes (mrt_render_batch,
    LPT-ordered), and per-scene launches of the plain megakernel, the
    regenerating megakernel, the wavefront and the per-scene autotuned
    choice (mrt_tune), and one batch call with every scene in its tuned
    form. Device time (CUDA events) summed over the calls."""
    import mrt
    import scenes
    specs = scenes.make_c3_specs()
    ctxs, scs = [], []
    t0 = time.perf_counter()
    for sp in specs:
        sc = scenes.make_c3_scene(sp)
        c = mrt.Context(sc.width, sc.height)
        c.build(sc)
        ctxs.append(c)
        scs.append(sc)
    build_s = time.perf_counter() - t0
    per_step = [max(1, sc.spp // 16) for sc in scs]
    paths_step = sum(sc.width * sc.height * k for sc, k in zip(scs, per_step))
    forms = {}
    clocks = Clocks(0)

    def per_scene(form):
        ms, launches = 0.0, 0
        for s in range(a.warmup + a.steps):
            step_ms = 0.0
            for c, sc, k in zip(ctxs, scs, per_step):
                st = c.render(k, seed=1, sample_base=s * k, form=form, max_bounces=sc.max_bounces)
                step_ms += st.ms
                if s >= a.warmup:
                    launches += st.kernel_launches
            if s >= a.warmup:
                ms += step_ms
        return ms, launches

    for c in ctxs:
        c.clear()
    ms, launches = 0.0, 0
    for s in range(a.warmup + a.steps):
        params = [dict(spp=k, sample_base=s * k, seed=1, max_bounces=sc.max_bounces)
                  for sc, k in zip(scs, per_step)]
        st = mrt.render_batch(ctxs, params)
        if s >= a.warmup:
            ms += st.ms
            launches += st.kernel_launches
    forms["batch"] = {"ms_per_step": ms / a.steps, "launches": launches}
    for name, fid in (("megakernel_plain", mrt.FORM_MEGAKERNEL_PLAIN), ("megakernel", mrt.FORM_MEGAKERNEL),
                      ("wavefront", mrt.FORM_WAVEFRONT)):
        ms, launches = per_scene(fid)
        forms[name] = {"ms_per_step": ms / a.steps, "launches": launches}
    picks = {}
    for c in ctxs:
        best = [e for e in c.tune(spp=1) if e["best"]][0]
        picks[best["form"]] = picks.get(best["form"], 0) + 1
    ms, launches = per_scene(mrt.FORM_AUTO)
    forms["autotuned"] = {"ms_per_step": ms / a.steps, "launches": launches, "tuner_picks": picks}
    # one batch call with each scene in its tuned form
    for c in ctxs:
        c.clear()
    ms, launches = 0.0, 0
    for s in range(a.warmup + a.steps):
        params = [dict(spp=k, sample_base=s * k, seed=1, max_bounces=sc.max_bounces, form=mrt.FORM_AUTO)
                  for sc, k in zip(scs, per_step)]
        st = mrt.render_batch(ctxs, params)
        if s >= a.warmup:
            ms += st.ms
            launches += st.kernel_launches
    forms["batch_autotuned"] = {"ms_per_step": ms / a.steps, "launches": launches, "tuner_picks": picks}
    clk = clocks.stop()
    for f in forms.values():
        f["value"] = paths_step / (f["ms_per_step"] / 1000.0) / 1e6
    best = max(forms, key=lambda k: forms[k]["value"])
    line = {
        "metric": METRIC, "value": forms[best]["value"], "unit": UNIT, "n_gpus": 1,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": forms[best]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator; the reference publishes no benchmark scene)",
        "config": {"workload": "c3: 64 scenes, 10k-2M triangles (log-uniform), 256^2-1024^2 pixels, "
                               "16-256 spp, depth 8-16, half 1024x512 HDRI half area light",
                   "paths_per_step": paths_step, "total_triangles": sum(sp["tris"] for sp in specs),
                   "parallelism": "single GPU"},
        "form": best, "forms": forms, "gpu_launches": forms[best]["launches"], "clocks": clk,
        "scene_build_s": build_s,
        "ratio_best_over_plain": forms[best]["value"] / forms["megakernel_plain"]["value"],
    }
    print(json.dumps(line), flush=True)
    for c in ctxs:
        c.close()
    return 0


WORKLOADS = {
    "c1": "c1: 1920x1080, 256 spp, depth 12, 1,310,720-triangle displaced geodesic sphere, "
          "16 materials, 2048x1024 RGBE sky with importance sampling",
    "q0": "q0: 320x240, 64 spp, depth 8, two cylinders, two cones, two hyperboloids, two spheres, "
          "ground plane, point light",
    "t0": "t0: 320x240, 64 spp, depth 8, image / checker / fallback textures, normal, roughness, metallic, "
          "ao and emission maps, alpha cut-outs",
}


def workload_config(a, sc) -> dict:
    return {"workload": WORKLOADS.get(a.config, a.config),
            "spp_per_step": a.spp_per_step,
            "l2": ("scene arrays (BVH, triangles, shading, sky tables) exceed the 126 MB L2"
                   if a.config not in ("q0", "t0") else "the scene (a few KB) stays in L2, as in any render of it; "
                   "each step traces new paths"),
            "parallelism": f"sample-parallel dp{a.gpus}"}


def main() -> int:
    a = parse()
    if a.impl == "reference":
        run_reference_arm(a)
        return 0
    if a.only_adjoint:
        print(json.dumps({"adjoint": adjoint_bench(0, a.adam_steps, a.adjoint_res)}), flush=True)
        return 0
    if a.config == "c3":
        return bench_c3(a)
    import distributed as D
    import mrt
    import scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        dist = tdist

    # CPU baseline first, before this process touches CUDA (it forks).
    cpu = None
    cpu_parity = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        runs = [x for x in (cpu_baseline(a.config, a.cpu_seconds, build=b) for b in ("fast", "parity"))
                if x is not None]
        cpu = max(runs, key=lambda x: x["mpaths_s"]) if runs else None
        cpu_parity = ([x for x in runs if x is not cpu] or [None])[0]

    sc = scenes.CONFIGS[a.config]()
    ctx = mrt.Context(sc.width, sc.height, device=local)
    t0 = time.perf_counter()
    ctx.build(sc)
    build_s = time.perf_counter() - t0
    if dist:
        # the library's own communicator (mrt_comm_init, NCCL): the frames of
        # all ranks are summed on rank 0 by mrt_reduce_frame
        cid = [mrt.comm_unique_id() if rank == 0 else None]
        dist.broadcast_object_list(cid, src=0)
        ctx.comm_init(cid[0], rank, world)
    npix = sc.width * sc.height
    spp = a.spp_per_step
    paths_per_step = npix * spp
    algo = json.loads((REPO / "oracle" / "algorithmic_bytes.json").read_text())
    # the progressive variant traces c2's scene (its extra gather bytes are not counted)
    bpp = algo["configs"][a.config.rstrip("p")]["bytes_per_path"]
    peaks = {}
    pk = REPO / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm = peaks.get("hbm_gbs", 6650.0)
    hbm_src = "of measured" if "hbm_gbs" in peaks else "of fallback"

    def barrier():
        if dist:
            dist.barrier()

    forms = {}
    form_ids = {"megakernel": mrt.FORM_MEGAKERNEL, "wavefront": mrt.FORM_WAVEFRONT,
                "megakernel_plain": mrt.FORM_MEGAKERNEL_PLAIN}
    clocks = Clocks(local)
    launches_total = 0
    best = None
    for name in a.forms.split(","):
        fid = form_ids[name]
        try:
            ctx.clear()
            for w in range(a.warmup):
                ctx.render(spp, seed=99, sample_base=w * spp, form=fid,
                           use_graph=1 if fid == mrt.FORM_WAVEFRONT else 0)
        except mrt.MRTError as e:
            forms[name] = {"error": str(e)[:200]}
            continue
        ctx.clear()
        barrier()
        ms = 0.0
        launches = 0
        step_ms = []
        base, _ = D.shard_samples(a.steps * spp * world, world, rank)
        for s in range(a.steps):
            st = ctx.render(spp, seed=1, sample_base=base + s * spp, form=fid,
                            use_graph=1 if fid == mrt.FORM_WAVEFRONT else 0)
            ms += st.ms
            step_ms.append(round(st.ms, 3))
            launches += st.kernel_launches
        if dist:
            # the frame of the job: one sum-reduce of the accumulators onto rank 0
            t_r = time.perf_counter()
            ctx.reduce_frame(0)
            ms += 1000.0 * (time.perf_counter() - t_r)
        barrier()
        t_max = ms
        if dist:
            import torch
            t = torch.tensor([ms], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_max = float(t.item())
        total_paths = paths_per_step * a.steps * world
        mps = total_paths / (t_max / 1000.0) / 1e6
        per_launch_ms = ms / max(launches, 1)
        forms[name] = {"value": mps, "ms_per_step": t_max / a.steps, "launches": launches,
                       "launch_ms": per_launch_ms, "step_ms": step_ms}
        if best is None or mps > forms[best]["value"]:
            best = name
        launches_total = launches
    clk = clocks.stop()
    if best is None:
        raise SystemExit("no render form ran: " + json.dumps(forms))

    # end to end through the C-ABI with host buffers, best form
    fid = form_ids[best]
    host = np.zeros(npix * 3, np.float64)
    cam = sc.desc().camera
    ctx.clear()
    barrier()
    t0 = time.perf_counter()
    for s in range(a.steps):
        ctx.set_camera(cam, sc.ior_all, sc.ambient_ratio)
        ctx.render(spp, seed=2, sample_base=rank * a.steps * spp + s * spp, form=fid,
                   use_graph=1 if fid == mrt.FORM_WAVEFRONT else 0)
        if dist:
            # every step's frame summed on rank 0 (mrt_reduce_frame), read
            # back there; the other ranks drop their consumed partial frame
            ctx.reduce_frame(0)
            if rank == 0:
                ctx.accumulate_double(host)
            else:
                ctx.clear()
        else:
            ctx.accumulate_double(host)
    barrier()
    e2e_s = time.perf_counter() - t0
    if dist:
        import torch
        t = torch.tensor([e2e_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = paths_per_step * a.steps * world / e2e_s / 1e6

    relmse = None
    if not a.no_relmse and world == 1:
        cap = a.relmse_cap_spp or (16384 if a.config == "c0" else 4096)
        relmse = convergence(ctx, sc, a.config, spp, forms, form_ids[best], cap)
    adjoint = None
    if not a.no_adjoint and world == 1:
        adjoint = adjoint_bench(local, a.adam_steps)

    f = forms[best]
    achieved = bpp * (paths_per_step / max(f["launches"] / a.steps, 1)) / (f["launch_ms"] / 1000.0) / 1e9
    # DRAM bytes per path of the form, from the ncu launch list summarised
    # in profiles/ (dram__bytes_read.sum + dram__bytes_write.sum over its
    # kernels), scaled to the paths of one launch like `achieved`
    traffic = None
    tf = REPO / "profiles" / "traffic.json"
    if tf.exists():
        t = json.loads(tf.read_text()).get(a.config, {}).get(best)
        if t:
            traffic = t["bytes_per_path"] * (paths_per_step / max(f["launches"] / a.steps, 1))
    line = {
        "metric": METRIC, "value": forms[best]["value"], "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": f["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator; the reference publishes no benchmark scene)",
        "config": workload_config(a, sc), "form": best, "forms": forms,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(__import__("ctypes").sizeof(mrt.Camera)),
                "d2h_bytes_per_step": int(npix * 3 * 4)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "peak_source": hbm_src,
                     "bytes_per_path": bpp},
        "gpu_launches": launches_total,
        "clocks": clk,
        "scene_build_s": build_s,
    }
    if relmse is not None:
        line["relmse"] = relmse
    if adjoint is not None:
        line["adjoint"] = adjoint
    if cpu is not None:
        line["cpu_baseline"] = {"value": cpu["mpaths_s"], "unit": UNIT, "cores": cpu["procs"],
                                "kind": "reference", "sample": cpu["sample"], "build": cpu["build"],
                                "other_build": None if cpu_parity is None else
                                {"value": cpu_parity["mpaths_s"], "build": cpu_parity["build"]}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        ctx.comm_destroy()
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
