"""Seeded synthetic radar scenes for FBME (2-D prefix-Fourier observations).

The reference ships no scene generator (its archived runner is missing), so
this module defines one.  A scene is a sparse complex image ``x`` on an
``N1 x N2`` grid, observed through the leading ``M1 x M2`` block of its
unnormalised 2-D DFT with complex white Gaussian noise:

    y = fft2(x)[:M1, :M2] + n,   E|n|^2 = mean|fft2(x)[:M1,:M2]|^2 / 10^(SNR/10)

which is the reference's observation model (torch_sbl/operators.py:23-30,
README "Input model").  All draws are float64 from ``numpy.random.default_rng``
and the observation is returned as complex64.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Scene:
    y: np.ndarray            # [M1, M2] complex64 observation
    x: np.ndarray            # [N1, N2] complex128 ground truth
    grid: tuple[int, int]
    noise_variance: float
    support: np.ndarray      # flat indices of the nonzero pixels


def _observe(x: np.ndarray, prefix, snr_db: float, rng) -> tuple[np.ndarray, float]:
    m1, m2 = prefix
    clean = np.fft.fft2(x)[:m1, :m2]
    noise_var = float(np.mean(np.abs(clean) ** 2) / 10.0 ** (snr_db / 10.0))
    noise = np.sqrt(noise_var / 2.0) * (
        rng.standard_normal(clean.shape) + 1j * rng.standard_normal(clean.shape)
    )
    return (clean + noise).astype(np.complex64), noise_var


def point_scene(grid, prefix, n_points: int, snr_db: float, seed: int,
                amplitude: str = "rayleigh") -> Scene:
    """``n_points`` scatterers at distinct uniform-random pixels.

    amplitude: "rayleigh" (|a| = sqrt(-2 ln U), sigma=1, uniform phase),
    "cn" (CN(0,1)), "lognormal" (exp(N(0,1)) magnitude, uniform phase).
    """
    rng = np.random.default_rng(seed)
    n1, n2 = grid
    x = np.zeros((n1, n2), np.complex128)
    idx = rng.choice(n1 * n2, size=n_points, replace=False)
    x.flat[idx] = _amplitudes(rng, n_points, amplitude)
    y, nv = _observe(x, prefix, snr_db, rng)
    return Scene(y, x, (n1, n2), nv, np.sort(idx))


def _amplitudes(rng, k: int, kind: str) -> np.ndarray:
    if kind == "cn":
        return (rng.standard_normal(k) + 1j * rng.standard_normal(k)) / np.sqrt(2.0)
    phase = np.exp(2j * np.pi * rng.random(k))
    if kind == "rayleigh":
        return np.sqrt(-2.0 * np.log1p(-rng.random(k))) * phase
    if kind == "lognormal":
        return np.exp(rng.standard_normal(k)) * phase
    raise ValueError(f"unknown amplitude law {kind!r}")


def cluster_scene(grid, prefix, seed: int, *, clusters: int = 10, per_cluster: int = 75,
                  isolated: int = 50, spread_px: float = 6.0, snr_db: float = 20.0) -> Scene:
    """Clustered scatterers: Gaussian offsets (std ``spread_px``) around
    uniform centres, rounded, wrapped and de-duplicated, plus isolated points.
    Log-normal magnitudes with uniform phase."""
    rng = np.random.default_rng(seed)
    n1, n2 = grid
    centres = np.stack([rng.integers(0, n1, clusters), rng.integers(0, n2, clusters)], 1)
    pts = []
    for c in centres:
        off = np.rint(rng.normal(0.0, spread_px, (per_cluster, 2))).astype(np.int64)
        p = (c[None, :] + off)
        p[:, 0] %= n1
        p[:, 1] %= n2
        pts.append(p[:, 0] * n2 + p[:, 1])
    flat = np.unique(np.concatenate(pts))
    rest = np.setdiff1d(np.arange(n1 * n2), flat)
    iso = rng.choice(rest, size=isolated, replace=False)
    idx = np.concatenate([flat, iso])
    x = np.zeros((n1, n2), np.complex128)
    x.flat[idx] = _amplitudes(rng, idx.size, "lognormal")
    y, nv = _observe(x, prefix, snr_db, rng)
    return Scene(y, x, (n1, n2), nv, np.sort(idx))


UNEVEN_GRIDS = ((128, 128), (192, 256), (256, 256), (384, 256))


def uneven_batch(batch_seed: int, n_scenes: int = 64) -> list[Scene]:
    """Batch of scenes with different grids and prefixes: grid drawn from
    ``UNEVEN_GRIDS``, prefix ratio per axis U[0.3, 0.7], sparsity U[1%, 3%]
    of the grid with CN(0,1) amplitudes, SNR U[5, 25] dB."""
    rng = np.random.default_rng(10_000 + batch_seed)
    out = []
    for i in range(n_scenes):
        g = UNEVEN_GRIDS[int(rng.integers(0, len(UNEVEN_GRIDS)))]
        r = rng.uniform(0.3, 0.7, 2)
        prefix = (max(1, int(round(r[0] * g[0]))), max(1, int(round(r[1] * g[1]))))
        k = max(1, int(round(rng.uniform(0.01, 0.03) * g[0] * g[1])))
        snr = float(rng.uniform(5.0, 25.0))
        out.append(point_scene(g, prefix, k, snr, int(rng.integers(0, 2**31 - 1)), "cn"))
    return out


def learned_scene(seed: int) -> Scene:
    """Training / evaluation scenes of the learned warm start: 256x256 grid,
    128x128 prefix, K ~ U{100..400} Rayleigh points, SNR ~ U[5, 25] dB."""
    rng = np.random.default_rng(7_000_000 + seed)
    k = int(rng.integers(100, 401))
    snr = float(rng.uniform(5.0, 25.0))
    return point_scene((256, 256), (128, 128), k, snr, seed, "rayleigh")


def config_scene(name: str, seed: int) -> Scene:
    """The named single-scene workloads.

    c1: 64x64 grid, 32x32 prefix, 40 CN(0,1) points, 20 dB.
    c2: 256x256 grid, 128x128 prefix, 200 Rayleigh points, 15 dB.
    c3: 512x512 grid, 256x192 prefix, clustered log-normal, 20 dB.
    """
    if name == "c1":
        return point_scene((64, 64), (32, 32), 40, 20.0, seed, "cn")
    if name == "c2":
        return point_scene((256, 256), (128, 128), 200, 15.0, seed, "rayleigh")
    if name == "c3":
        return cluster_scene((512, 512), (256, 192), seed)
    raise ValueError(name)


def nmse_db(x_hat: np.ndarray, x: np.ndarray) -> float:
    """Raw NMSE in dB, no gain alignment."""
    num = float(np.sum(np.abs(np.asarray(x_hat) - x) ** 2))
    den = float(np.sum(np.abs(x) ** 2))
    return 10.0 * np.log10(max(num, 1e-300) / den)
