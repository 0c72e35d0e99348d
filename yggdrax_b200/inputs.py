"""Seeded synthetic point sets for the pipeline's workloads.

All generators draw with ``numpy.random.Generator(PCG64(seed))`` in float64
and return float32 ``(positions (N, 3), masses (N,))`` numpy arrays.
"""

from __future__ import annotations

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def uniform_cube(n: int, seed: int = 0, *, lo: float = -1.0, hi: float = 1.0,
                 mass_range=(0.5, 1.5)):
    """Uniform in [lo, hi]^3, masses uniform in mass_range."""
    rng = _rng(seed)
    pos = rng.uniform(lo, hi, size=(n, 3))
    mass = rng.uniform(mass_range[0], mass_range[1], size=n)
    return pos.astype(np.float32), mass.astype(np.float32)


def _plummer_radii(rng: np.random.Generator, n: int, a: float, rmax: float) -> np.ndarray:
    """Inverse-CDF Plummer radii r = a / sqrt(X^(-2/3) - 1), rejecting r > rmax."""
    out = np.empty(0)
    while out.shape[0] < n:
        m = int((n - out.shape[0]) * 1.05) + 16
        x = rng.uniform(0.0, 1.0, size=m)
        x = x[x > 0]
        r = a / np.sqrt(x ** (-2.0 / 3.0) - 1.0)
        out = np.concatenate([out, r[r <= rmax]])
    return out[:n]


def _directions(rng: np.random.Generator, n: int) -> np.ndarray:
    cos_t = rng.uniform(-1.0, 1.0, size=n)
    phi = rng.uniform(0.0, 2.0 * np.pi, size=n)
    sin_t = np.sqrt(1.0 - cos_t * cos_t)
    return np.stack([sin_t * np.cos(phi), sin_t * np.sin(phi), cos_t], axis=1)


def plummer(n: int, seed: int = 1, *, a: float = 1.0, rmax: float = 20.0):
    """Plummer sphere (scale radius a, truncated at rmax), equal masses 1/N."""
    rng = _rng(seed)
    r = _plummer_radii(rng, n, a, rmax)
    pos = r[:, None] * _directions(rng, n)
    mass = np.full(n, 1.0 / n)
    return pos.astype(np.float32), mass.astype(np.float32)


def plummer_clumps(n: int, seed: int = 2, *, clumps: int = 64, box: float = 10.0,
                   a_range=(0.05, 0.5)):
    """Mixture of Plummer clumps: centres uniform in [-box, box]^3, scale radii
    log-uniform in a_range, each truncated at 20a; lognormal(0, 1) masses."""
    rng = _rng(seed)
    centres = rng.uniform(-box, box, size=(clumps, 3))
    scales = np.exp(rng.uniform(np.log(a_range[0]), np.log(a_range[1]), size=clumps))
    per = np.full(clumps, n // clumps)
    per[: n - per.sum()] += 1
    parts = []
    for c in range(clumps):
        r = _plummer_radii(rng, int(per[c]), scales[c], 20.0 * scales[c])
        parts.append(centres[c] + r[:, None] * _directions(rng, int(per[c])))
    pos = np.concatenate(parts, axis=0)
    mass = rng.lognormal(0.0, 1.0, size=n)
    return pos.astype(np.float32), mass.astype(np.float32)


def batched_sets(sets: int = 4096, seed: int = 3, *, lo: int = 256, hi: int = 65536):
    """Independent point sets of uneven size, stored back to back: set sizes
    ``floor(exp(U[ln lo, ln hi]))``, even-numbered sets uniform in [-1, 1]^3,
    odd-numbered sets Plummer spheres (a = 1, r <= 20); unit masses.
    Returns ``(positions (N, 3), masses (N,), offsets (sets + 1,) int64)``."""
    rng = _rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), size=sets))).astype(np.int64)
    sizes = np.maximum(sizes, 1)
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    pos = np.empty((int(offsets[-1]), 3), np.float32)
    for s in range(sets):
        n = int(sizes[s])
        if s % 2 == 0:
            p = rng.uniform(-1.0, 1.0, size=(n, 3))
        else:
            p = _plummer_radii(rng, n, 1.0, 20.0)[:, None] * _directions(rng, n)
        pos[offsets[s]:offsets[s + 1]] = p
    return pos, np.ones(pos.shape[0], np.float32), offsets


__all__ = ["uniform_cube", "plummer", "plummer_clumps", "batched_sets"]
