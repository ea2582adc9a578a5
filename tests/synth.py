"""Seeded synthetic planes shaped like the workloads the reference is measured on
(no dataset is involved). Seeds follow numpy.random.default_rng([config, clip, frame])."""
from __future__ import annotations

import numpy as np
from scipy.ndimage import gaussian_filter


def textured(h: int, w: int, seed, lo: float, hi: float, sd_px: float = 3.0) -> np.ndarray:
    """Band-limited texture (Gaussian-filtered white noise) rescaled to [lo, hi]."""
    rng = np.random.default_rng(seed)
    t = gaussian_filter(rng.standard_normal((h, w)), sd_px)
    t = (t - t.min()) / max(np.ptp(t), 1e-12)
    return lo + (hi - lo) * t


def gradient_sinusoid(h: int, w: int, seed) -> np.ndarray:
    """Smooth gradient plus sinusoids with periods 7-40 px, in [16, 235]."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    img = 0.5 * (x / max(w - 1, 1)) + 0.3 * (y / max(h - 1, 1))
    for _ in range(4):
        px, py = rng.uniform(7, 40, 2)
        img += 0.15 * np.sin(2 * np.pi * (x / px + y / py) + rng.uniform(0, 2 * np.pi))
    img = (img - img.min()) / max(np.ptp(img), 1e-12)
    return 16 + 219 * img


def to_format(v: np.ndarray, bits: int, floating: bool, noise_sd: float, seed) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = v + rng.standard_normal(v.shape) * noise_sd
    if floating:
        return v.astype(np.float32)
    peak = (1 << bits) - 1
    v = np.clip(np.round(v), 0, peak)
    return v.astype(np.uint8 if bits == 8 else np.uint16)


def plane(h, w, bits=8, floating=False, seed=(0, 0, 0), kind="texture"):
    """One seeded plane in the sample units of the format."""
    if floating:
        base = textured(h, w, seed, 0.0, 1.0)
        return to_format(base, bits, True, 0.02, (*seed, 1))
    peak = (1 << bits) - 1
    if kind == "gradient":
        base = gradient_sinusoid(h, w, seed) * (peak / 255.0)
    else:
        base = textured(h, w, seed, 0.06 * peak, 0.92 * peak)
    return to_format(base, bits, False, 0.02 * peak, (*seed, 1))


def noisy_patches(n: int, size: int, seed):
    """Differentiable-training workload: clean = band-limited texture in [0, 1]; noisy =
    clean + coloured Gaussian noise whose amplitude spectrum follows a seeded random radial
    curve, with the noise sd drawn from U[0.01, 0.05] per patch. Returns (noisy, clean),
    float32 [n, size, size]."""
    rng = np.random.default_rng(seed)
    clean = np.stack([textured(size, size, (*np.atleast_1d(seed), 100, i), 0.0, 1.0) for i in range(n)])
    fy = np.fft.fftfreq(size)[:, None]
    fx = np.fft.rfftfreq(size)[None, :]
    r = np.sqrt(fx * fx + fy * fy) / np.sqrt(0.5)
    noisy = np.empty_like(clean)
    for i in range(n):
        knots = rng.uniform(0.2, 1.0, 6)
        curve = np.interp(r, np.linspace(0, 1, 6), knots)
        spec = np.fft.rfft2(rng.standard_normal((size, size))) * curve
        noise = np.fft.irfft2(spec, s=(size, size))
        noise *= rng.uniform(0.01, 0.05) / max(noise.std(), 1e-12)
        noisy[i] = clean[i] + noise
    return noisy.astype(np.float32), clean.astype(np.float32)
