"""Seeded synthetic particle sets for the treecode workloads.

Every generator draws from SplitMix64 (Steele, Lea & Flood, "Fast splittable
pseudorandom number generators", OOPSLA 2014), evaluated counter-style so that
element ``i`` of stream ``s`` under seed ``k`` is a pure function of (k, s, i):
the same inputs come out of numpy here and of any other implementation of the
same three-line mixer. Doubles are the top 53 bits scaled by 2**-53.

The reference drivers draw points from an unseeded ``std::mt19937``
(examples/example_poisson_3d.cpp:44-48); seeded generators make runs
reproducible and let fixtures be regenerated.
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def u64(seed: int, stream: int, n: int, offset: int = 0) -> np.ndarray:
    """n raw 64-bit outputs of stream ``stream`` under ``seed``."""
    with np.errstate(over="ignore"):
        base = _mix(np.array([(seed * 0x9E3779B97F4A7C15 + stream * 0xD1B54A32D192ED03) & (2**64 - 1)],
                             dtype=np.uint64))[0]
        i = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        return _mix(base + i * _GOLDEN)


def uniform(seed: int, stream: int, n: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
    u = (u64(seed, stream, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return lo + (hi - lo) * u


def normal(seed: int, stream: int, n: int) -> np.ndarray:
    """Standard normals by Box-Muller on two uniform streams."""
    u1 = uniform(seed, 2 * stream + 1000, n)
    u2 = uniform(seed, 2 * stream + 1001, n)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)


def uniform_box(seed: int, n: int, dim: int, lo: float, hi: float, q_lo: float = -1.0, q_hi: float = 1.0):
    """Points uniform in [lo,hi]^dim, charges uniform in [q_lo,q_hi]."""
    pts = tuple(uniform(seed, d, n, lo, hi) for d in range(dim))
    q = uniform(seed, 10, n, q_lo, q_hi)
    return pts, q


def plummer(seed: int, n: int, scale: float = 0.1, rmax: float = 2.0):
    """Plummer-sphere positions (scale radius ``scale``) truncated at r <= rmax by
    rejection; charges uniform in [0,1]. Radius by inverse CDF
    r = a / sqrt(u^(-2/3) - 1); direction uniform on the sphere."""
    out = []
    got, block, off = 0, max(1024, int(n * 1.1)), 0
    while got < n:
        uu = uniform(seed + off, 20, block)
        r = scale / np.sqrt(np.power(np.clip(uu, 1e-300, 1.0), -2.0 / 3.0) - 1.0 + 1e-300)
        cz = uniform(seed + off, 21, block, -1.0, 1.0)
        ph = uniform(seed + off, 22, block, 0.0, 2.0 * np.pi)
        keep = r <= rmax
        s = np.sqrt(1.0 - cz * cz)
        xyz = np.stack([r * s * np.cos(ph), r * s * np.sin(ph), r * cz], axis=1)[keep]
        out.append(xyz)
        got += len(xyz)
        off += 1
    xyz = np.concatenate(out)[:n]
    q = uniform(seed, 23, n, 0.0, 1.0)
    return (xyz[:, 0].copy(), xyz[:, 1].copy(), xyz[:, 2].copy()), q


def sphere_surface(seed: int, n: int):
    """Points uniform in area on the unit sphere (normalised Gaussians);
    strengths uniform in [-1,1]."""
    g = np.stack([normal(seed, d, n) for d in range(3)], axis=1)
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    q = uniform(seed, 30, n, -1.0, 1.0)
    return (g[:, 0].copy(), g[:, 1].copy(), g[:, 2].copy()), q


def gaussian_mixture(seed: int, n: int):
    """Mixture of 1-8 isotropic Gaussians (sigma in [0.02, 0.2], centres in the
    unit cube), rejected to [0,1]^3; standard-normal charges."""
    k = 1 + int(uniform(seed, 40, 1)[0] * 8)
    centres = np.stack([uniform(seed, 41 + d, k, 0.0, 1.0) for d in range(3)], axis=1)
    sig = uniform(seed, 44, k, 0.02, 0.2)
    out, got, off = [], 0, 0
    while got < n:
        m = max(1024, int(1.3 * (n - got)))
        comp = np.minimum((uniform(seed + 7919 * off, 45, m) * k).astype(np.int64), k - 1)
        p = centres[comp] + sig[comp, None] * np.stack([normal(seed + 7919 * off, 50 + d, m) for d in range(3)], 1)
        p = p[np.all((p >= 0.0) & (p <= 1.0), axis=1)]
        out.append(p)
        got += len(p)
        off += 1
    xyz = np.concatenate(out)[:n]
    q = normal(seed, 60, n)
    return (xyz[:, 0].copy(), xyz[:, 1].copy(), xyz[:, 2].copy()), q
