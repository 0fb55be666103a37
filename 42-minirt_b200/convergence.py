"""Converged-radiance comparison of a render with a reference render whose
per-pixel noise is known.

The reference side is a converged-radiance fixture (tests/golden/conv_*.npz):
the reference CPU renderer's per-pixel mean at 4096 samples per pixel over a
pixel set, the variance of that mean (from batch means), and the image mean
of each batch. relMSE follows the metric's definition,
mean((x - r)^2 / (r^2 + 0.01)) over pixels and channels.

Both images are noisy, so E[(x - r)^2] = bias^2 + var_x + var_r per pixel.
  relmse_raw        the plain relMSE of x against r;
  relmse_converged  relMSE of x against the converged image the reference
                    estimates: the raw terms minus var_r (an unbiased estimate
                    of E[(x - mu)^2] when r is unbiased for mu);
  relmse_bias       relMSE of the expectations: minus var_x too (an unbiased
                    estimate of the squared bias term, may come out negative).
Per-pixel z-scores (x - r) / sqrt(var_x + var_r + floor^2), floor =
Z_FLOOR_REL |r| + Z_FLOOR_ABS (rounding, for pixels without noise).
The image-mean bias test compares the two image means per channel against
their standard error, taken from the spread of the batch image means (pixels
of one reference batch share their sample offsets, so per-pixel variances
would understate it).
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

EPS = 1e-2
# Per-pixel z-scores get a precision floor in their denominator: a pixel can
# have (near) zero variance on both sides (every sample sees the same sky
# texel or nothing), where the FP32 kernel and the FP64 reference still differ
# by rounding. 1e-4 relative (about 1,700 FP32 ulps) plus 1e-6 absolute is far
# below any shading difference a shifted or blurred image would show.
Z_FLOOR_REL = 1e-4
Z_FLOOR_ABS = 1e-6


def load_fixture(path: str | Path) -> dict:
    z = np.load(path, allow_pickle=False)
    out = {k: z[k] for k in z.files if k != "meta"}
    out.update(json.loads(str(z["meta"])))
    return out


def pixel_values(img: np.ndarray, pixels: np.ndarray) -> np.ndarray:
    """(n, 3) values of an (H, W, 3) image at linear pixel indices y * W + x."""
    h, w = img.shape[:2]
    return img.reshape(h * w, -1)[pixels, :3]


def relmse(x: np.ndarray, r: np.ndarray) -> float:
    return float(np.mean((x - r) ** 2 / (r ** 2 + EPS)))


def relmse_converged(x: np.ndarray, r: np.ndarray, var_r: np.ndarray) -> float:
    return float(np.mean(((x - r) ** 2 - var_r) / (r ** 2 + EPS)))


def batch_summary(batch_means: np.ndarray) -> dict:
    """Per-pixel mean, variance of that mean and per-batch image means of a
    render split into batches: batch_means (B, n, 3) or (B, H, W, 3)."""
    bm = np.asarray(batch_means, np.float64)
    bm = bm.reshape(bm.shape[0], -1, bm.shape[-1])[..., :3]
    return {"mean": bm.mean(0), "var_mean": bm.var(0, ddof=1) / bm.shape[0],
            "batch_image_mean": bm.mean(1)}


def compare(x: np.ndarray, var_x: np.ndarray, batch_means_x: np.ndarray, ref: dict) -> dict:
    """Statistics of a render (per-pixel mean x, variance of that mean var_x,
    per-batch image means) against a converged-radiance fixture."""
    r, var_r = ref["mean"].astype(np.float64), ref["var_mean"].astype(np.float64)
    w = 1.0 / (r ** 2 + EPS)
    d2 = (x - r) ** 2
    out = {
        "pixels": int(len(r)),
        "relmse_raw": float(np.mean(d2 * w)),
        "relmse_noise_ref": float(np.mean(var_r * w)),
        "relmse_noise_ours": float(np.mean(var_x * w)),
        "relmse_converged": float(np.mean((d2 - var_r) * w)),
        "relmse_bias": float(np.mean((d2 - var_r - var_x) * w)),
        # standard error of relmse_bias from the spread of its per-pixel terms
        "relmse_bias_se": float(np.std((d2 - var_r - var_x) * w) / np.sqrt(d2.size)),
    }
    bx = np.asarray(batch_means_x, np.float64)
    br = np.asarray(ref["batch_image_mean"], np.float64)
    se = np.sqrt(bx.var(0, ddof=1) / len(bx) + br.var(0, ddof=1) / len(br))
    diff = bx.mean(0) - br.mean(0)
    out["image_mean_ours"] = bx.mean(0).tolist()
    out["image_mean_ref"] = br.mean(0).tolist()
    out["image_mean_z"] = (diff / np.maximum(se, 1e-30)).tolist()
    floor = Z_FLOOR_REL * np.abs(r) + Z_FLOOR_ABS
    z = (x - r) / np.sqrt(var_x + var_r + floor ** 2)
    out["pixel_z_rms"] = float(np.sqrt(np.mean(z ** 2)))
    out["pixel_z_gt5"] = float(np.mean(np.abs(z) > 5))
    # the bias relMSE over the pixels whose every channel is within 5
    # standard errors (the outliers are bounded separately by pixel_z_gt5):
    # a handful of firefly pixels, whose variance a few batch means cannot
    # estimate, would otherwise decide it
    keep = np.all(np.abs(z) <= 5, axis=-1) if z.ndim > 1 else np.abs(z) <= 5
    tb = ((d2 - var_r - var_x) * w)[keep]
    out["relmse_bias_inliers"] = float(np.mean(tb)) if tb.size else 0.0
    out["relmse_bias_inliers_se"] = float(np.std(tb) / np.sqrt(max(tb.size, 1)))
    return out
