"""Seeded synthetic inputs standing in for the reference's sample data.

The reference's benchmark volumes (JHU isotropic turbulence, Utah DEM) are not
part of the reference tree, so the workloads use seeded synthetic fields of the
same shapes and statistics:

* ``turbulence_field``: sum of random-phase Fourier modes with amplitude
  |k|^(-5/3), integer wave vectors drawn uniformly in the cube and rejection
  sampled to 1 <= |k| <= kmax, phases uniform in [0, 2*pi); normalised to zero
  mean and unit standard deviation.  Evaluated exactly (float64) by placing the
  modes on an FFT grid and taking the inverse transform.
* ``fbm_heightfield``: fractional-Brownian value noise (10 octaves, lacunarity
  2, gain 2^-H) scaled to a height range and rounded to int16.
* ``brick_set``: uneven bricks cut at random offsets from seeded fields.

All generators use NumPy's PCG64 ``default_rng(seed)``.
"""
from __future__ import annotations

import numpy as np

SEED_C0 = 1000
SEED_C1 = 1001
SEED_C2 = (1002, 1003, 1004)
SEED_C3 = 1005
SEED_C4 = 1006


def turbulence_field(n: int, modes: int, kmax: int, seed: int) -> np.ndarray:
    """n^3 float32 field, sum of ``modes`` random-phase |k|^(-5/3) modes."""
    rng = np.random.default_rng(seed)
    ks = []
    while len(ks) < modes:
        k = rng.integers(-kmax, kmax + 1, size=3)
        r = float(np.sqrt((k * k).sum()))
        if 1.0 <= r <= kmax:
            ks.append(k)
    ks = np.array(ks, dtype=np.int64)
    phase = rng.uniform(0.0, 2.0 * np.pi, size=modes)
    amp = np.sqrt((ks * ks).sum(axis=1)).astype(np.float64) ** (-5.0 / 3.0)
    spec = np.zeros((n, n, n), dtype=np.complex128)
    # index order (z, y, x); k = (kx, ky, kz)
    np.add.at(spec, (ks[:, 2] % n, ks[:, 1] % n, ks[:, 0] % n), amp * np.exp(1j * phase))
    f = np.fft.ifftn(spec).real * float(n) ** 3
    f -= f.mean()
    f /= f.std()
    return np.ascontiguousarray(f.astype(np.float32))


def fbm_heightfield(n: int, seed: int, octaves: int = 10, hurst: float = 0.8,
                    lo: float = -2000.0, hi: float = 8000.0) -> np.ndarray:
    """n x n int16 terrain: fBm of smoothstep-interpolated value noise."""
    rng = np.random.default_rng(seed)
    gain = 2.0 ** (-hurst)
    acc = np.zeros((n, n), dtype=np.float64)
    amp = 1.0
    for o in range(octaves):
        cells = 2 << o                       # lattice cells across the tile
        lat = rng.uniform(-1.0, 1.0, size=(cells + 1, cells + 1))
        t = np.arange(n, dtype=np.float64) * cells / n
        i0 = np.floor(t).astype(np.int64)
        f = t - i0
        f = f * f * (3.0 - 2.0 * f)
        i1 = i0 + 1
        fy = f[:, None]
        fx = f[None, :]
        v00 = lat[i0[:, None], i0[None, :]]
        v01 = lat[i0[:, None], i1[None, :]]
        v10 = lat[i1[:, None], i0[None, :]]
        v11 = lat[i1[:, None], i1[None, :]]
        top = v00 + (v01 - v00) * fx
        bot = v10 + (v11 - v10) * fx
        acc += amp * (top + (bot - top) * fy)
        amp *= gain
    acc = (acc - acc.min()) / (acc.max() - acc.min())
    return np.rint(lo + acc * (hi - lo)).astype(np.int16)


def brick_set(count: int, seed: int, edges=(16, 24, 32, 48, 64), source_n: int = 256,
              source_fields: int = 4, q_lo: float = 0.002, q_hi: float = 0.05, cubic: bool = False):
    """Uneven bricks cut from seeded k^(-5/3) fields.

    Returns (bricks, q) where bricks is a list of float32 arrays shaped
    (z, y, x) and q the per-brick quantization step (log-uniform in
    [q_lo, q_hi] times the field's unit std)."""
    rng = np.random.default_rng(seed)
    srcs = [turbulence_field(source_n, 1024, 64, seed + 1 + j) for j in range(source_fields)]
    bricks, q = [], []
    for _ in range(count):
        if cubic:
            e = int(rng.choice(edges))
            ex = ey = ez = e
        else:
            ex, ey, ez = (int(v) for v in rng.choice(edges, size=3))
        s = srcs[int(rng.integers(0, source_fields))]
        ox = int(rng.integers(0, source_n - ex + 1))
        oy = int(rng.integers(0, source_n - ey + 1))
        oz = int(rng.integers(0, source_n - ez + 1))
        bricks.append(np.ascontiguousarray(s[oz:oz + ez, oy:oy + ey, ox:ox + ex]))
        q.append(float(np.exp(rng.uniform(np.log(q_lo), np.log(q_hi)))))
    return bricks, np.array(q, dtype=np.float32)


def psnr(orig: np.ndarray, recon: np.ndarray) -> float:
    """20*log10((max-min)/RMSE) in float64 (reference tools/imgtools.h:32-44,114-143)."""
    o = orig.astype(np.float64)
    r = recon.astype(np.float64)
    rmse = float(np.sqrt(np.mean((o - r) ** 2)))
    rng = float(o.max() - o.min())
    if rmse == 0.0:
        return float("inf")
    return 20.0 * np.log10(rng / rmse)
