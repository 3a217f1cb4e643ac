"""Statistical image comparison shared by the parity tests.

Two converged estimates of one image agree when

* each channel's image mean differs by at most 3 standard errors of the
  difference, and
* the relative RMSE between them (the reference's ``image_error_metrics``,
  ordinarylight/validation/_core.py:249-263) is below the stated tolerance
  once both sides' Monte Carlo noise is removed:
  E[rmse^2] = bias^2 + mean(sem_a^2) + mean(sem_b^2), so
  bias = sqrt(max(rmse^2 - noise^2, 0)), relative to the reference image's
  RMS value.
"""

from __future__ import annotations

import numpy as np


def image_error_metrics(reference, candidate):
    reference = np.asarray(reference, np.float64)[..., :3]
    candidate = np.asarray(candidate, np.float64)[..., :3]
    diff = candidate - reference
    rmse = float(np.sqrt(np.mean(diff * diff)))
    scale = float(np.sqrt(np.mean(reference * reference)))
    return {"rmse": rmse, "relative_rmse": rmse / max(scale, 1e-8), "mae": float(np.mean(np.abs(diff)))}


def batch_estimate(batches):
    """(mean, per-pixel sem, per-channel image-mean se) of K independent
    equally weighted batch images (K, h, w, 3)."""
    b = np.asarray(batches, np.float64)[..., :3]
    k = len(b)
    image_means = b.reshape(k, -1, 3).mean(axis=1)
    return b.mean(axis=0), b.std(axis=0, ddof=1) / np.sqrt(k), image_means.std(axis=0, ddof=1) / np.sqrt(k)


def compare(ref_mean, ref_sem, ref_image_se, mean, sem, image_se, *, tolerance=0.01, label=""):
    """Assert the two agreement criteria; returns (image-mean differences,
    their 3-SE bounds, noise-corrected relative RMSE, raw relative RMSE)."""
    ref_mean = np.asarray(ref_mean, np.float64)
    mean = np.asarray(mean, np.float64)
    diff = np.abs(ref_mean.reshape(-1, 3).mean(axis=0) - mean.reshape(-1, 3).mean(axis=0))
    bound = 3.0 * np.sqrt(np.asarray(ref_image_se) ** 2 + np.asarray(image_se) ** 2)
    raw = image_error_metrics(ref_mean, mean)
    scale = float(np.sqrt(np.mean(ref_mean ** 2)))
    noise = float(np.sqrt(np.mean(np.asarray(ref_sem, np.float64) ** 2 + np.asarray(sem, np.float64) ** 2)))
    bias = float(np.sqrt(max(raw["rmse"] ** 2 - noise ** 2, 0.0))) / scale
    assert np.all(diff <= bound), f"{label}: image means differ by {diff}, 3 SE = {bound}"
    assert bias < tolerance, (f"{label}: noise-corrected relative RMSE {bias:.4f} (raw {raw['relative_rmse']:.4f}, "
                              f"noise {noise / scale:.4f})")
    return diff, bound, bias, raw["relative_rmse"]


def oracle_image_se(sem):
    """Per-channel standard error of the image mean of an estimate whose
    pixels are independent, from its per-pixel standard errors."""
    s = np.asarray(sem, np.float64).reshape(-1, 3)
    return np.sqrt(np.sum(s * s, axis=0)) / len(s)
