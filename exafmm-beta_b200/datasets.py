"""Seeded body generators for the benchmark workloads, plus the reference's own.

The reference's generators (include/dataset.h) draw with drand48 from fixed
shapes ([-pi, pi]^3 cube, radius-pi sphere, Plummer scaled by 3*pi/16).  The
workloads this engine is measured on use different shapes, so they are
generated here with numpy's PCG64 from an explicit seed and handed, as the
same (n, 4) array, to both the GPU engine and the CPU checkers.

Every generator returns float64 (n, 4): x, y, z, charge.
"""
from __future__ import annotations

import numpy as np


def _zero_mean(q: np.ndarray) -> np.ndarray:
    return q - q.mean()


def cube(n: int, seed: int = 1, charge: str = "uniform") -> np.ndarray:
    """Uniform in [-1, 1]^3; charges U[-1, 1] shifted to zero net charge."""
    rng = np.random.default_rng(seed)
    x = np.empty((n, 4))
    x[:, :3] = rng.uniform(-1.0, 1.0, (n, 3))
    x[:, 3] = _zero_mean(rng.uniform(-1.0, 1.0, n)) if n else 0.0
    return x


def sphere(n: int, seed: int = 1) -> np.ndarray:
    """Uniform on the unit sphere surface (normalized Gaussians); charges U[-1, 1]."""
    rng = np.random.default_rng(seed)
    g = rng.normal(size=(n, 3))
    x = np.empty((n, 4))
    x[:, :3] = g / np.linalg.norm(g, axis=1)[:, None]
    x[:, 3] = rng.uniform(-1.0, 1.0, n)
    return x


def plummer(n: int, seed: int = 2, rmax: float = 20.0, scale: float = 1.0) -> np.ndarray:
    """Plummer sphere: radius by the inverse CDF (U^(-2/3) - 1)^(-1/2) (the form of
    include/dataset.h:121), rejected beyond rmax, isotropic directions; equal
    charges 1/n."""
    rng = np.random.default_rng(seed)
    out = np.empty((0, 3))
    while len(out) < n:
        m = int((n - len(out)) * 1.05) + 16
        u = rng.uniform(size=m)
        with np.errstate(divide="ignore"):
            r = scale / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        r = r[np.isfinite(r) & (r <= rmax * scale)]
        g = rng.normal(size=(len(r), 3))
        out = np.vstack([out, g / np.linalg.norm(g, axis=1)[:, None] * r[:, None]])
    x = np.empty((n, 4))
    x[:, :3] = out[:n]
    x[:, 3] = 1.0 / n
    return x


def water_box(n_waters: int, seed: int = 5, density: float = 0.0334):
    """Rigid 3-site waters (O -0.834, H +0.417, O-H 0.9572 A, H-O-H 104.52 deg) at
    random positions and orientations in a cubic box of edge L = (n/density)^(1/3),
    mapped to [-L/2, L/2]^3.  Returns (xyzq, L)."""
    rng = np.random.default_rng(seed)
    L = (n_waters / density) ** (1.0 / 3.0)
    O = rng.uniform(-L / 2, L / 2, (n_waters, 3))
    # random rotation per molecule from normalized quaternions
    q = rng.normal(size=(n_waters, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    w, a, b, c = q.T
    R = np.stack([
        np.stack([1 - 2 * (b * b + c * c), 2 * (a * b - c * w), 2 * (a * c + b * w)], -1),
        np.stack([2 * (a * b + c * w), 1 - 2 * (a * a + c * c), 2 * (b * c - a * w)], -1),
        np.stack([2 * (a * c - b * w), 2 * (b * c + a * w), 1 - 2 * (a * a + b * b)], -1),
    ], 1)
    d, half = 0.9572, np.deg2rad(104.52) / 2
    h1 = np.array([d * np.sin(half), 0.0, d * np.cos(half)])
    h2 = np.array([-d * np.sin(half), 0.0, d * np.cos(half)])
    H1 = O + R @ h1
    H2 = O + R @ h2
    pos = np.stack([O, H1, H2], 1).reshape(-1, 3)
    pos = (pos + L / 2) % L - L / 2  # wrap into the box
    chg = np.tile([-0.834, 0.417, 0.417], n_waters)
    return np.c_[pos, chg], L


def log_uniform_sizes(count: int, lo: int, hi: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)


def strided_sample(n: int, k: int) -> np.ndarray:
    """Dataset::sampleBodies (include/dataset.h:290-298): every (n // k)-th body."""
    if k >= n:
        return np.arange(n)
    return np.arange(k) * (n // k)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """Verify::getDif*/getNrm* (include/verify.h:42-107): sqrt(sum|a-b|^2 / sum|b|^2),
    b being the reference argument."""
    num = float(np.sum((np.asarray(a) - np.asarray(b)) ** 2))
    den = float(np.sum(np.asarray(b) ** 2))
    return float(np.sqrt(num / den)) if den > 0 else float(np.sqrt(num))
