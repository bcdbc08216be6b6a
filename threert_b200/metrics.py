"""Image error as the reference reports it: renderer/src/compare.rs `compare_region` (8-bit sRGB images, linearised,
to CIE Lab, the per-pixel ΔE (CIE76) with its mean, 95th and 99th percentiles).

The pass writes HDR radiance; the reference's own display transform (post.rs: auto exposure, local exposure, tone
curve) is not part of it, so images are brought to 8-bit sRGB here by a fixed exposure (by default the one that maps
the reference image's mean luminance to 0.18), a clamp and the sRGB curve, the same for both images.
"""
from __future__ import annotations

import numpy as np

LUM = np.array([0.2126, 0.7152, 0.0722])


def to_srgb8(rgb: np.ndarray, exposure: float) -> np.ndarray:
    c = np.clip(np.nan_to_num(np.asarray(rgb, np.float64) * exposure, nan=0.0, posinf=1.0, neginf=0.0), 0.0, 1.0)
    s = np.where(c <= 0.0031308, 12.92 * c, 1.055 * np.power(c, 1.0 / 2.4) - 0.055)
    return np.clip(np.round(s * 255.0), 0, 255).astype(np.uint8)


def _linear(c8: np.ndarray) -> np.ndarray:
    # compare.rs:27-30
    c = c8.astype(np.float64) / 255.0
    return np.where(c <= 0.04045, c / 12.92, np.power((c + 0.055) / 1.055, 2.4))


def lab(c: np.ndarray) -> np.ndarray:
    """compare.rs:135-142 lab: linear sRGB (..., 3) to CIE L*a*b* (D65)."""
    x = (0.4124 * c[..., 0] + 0.3576 * c[..., 1] + 0.1805 * c[..., 2]) / 0.95047
    y = 0.2126 * c[..., 0] + 0.7152 * c[..., 1] + 0.0722 * c[..., 2]
    z = (0.0193 * c[..., 0] + 0.1192 * c[..., 1] + 0.9505 * c[..., 2]) / 1.08883
    f = lambda t: np.where(t > 0.008856, np.cbrt(t), 7.787 * t + 16.0 / 116.0)
    fx, fy, fz = f(x), f(y), f(z)
    return np.stack([116.0 * fy - 16.0, 500.0 * (fx - fy), 200.0 * (fy - fz)], -1)


def exposure_for(reference: np.ndarray) -> float:
    m = float((np.nan_to_num(np.asarray(reference, np.float64)) @ LUM).mean())
    return 0.18 / m if m > 0 else 1.0


def delta_e(reference: np.ndarray, test: np.ndarray, exposure: float | None = None) -> dict:
    """ΔE (CIE76) of `test` against `reference`, both (h, w, 3) linear radiance: mean, p95, p99 (compare.rs:43-93)."""
    k = exposure_for(reference) if exposure is None else exposure
    la, lb = lab(_linear(to_srgb8(reference, k))), lab(_linear(to_srgb8(test, k)))
    de = np.sqrt(((la - lb) ** 2).sum(-1)).ravel()
    s = np.sort(de)
    n = len(s)
    return {"mean": float(de.mean()), "p95": float(s[int(n * 0.95)]), "p99": float(s[min(int(n * 0.99), n - 1)]),
            "exposure": k}
