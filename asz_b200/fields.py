"""Seeded synthetic float32 fields with the shapes and statistics of the benchmark workloads.

The reference was measured on external scientific datasets, which are not available here. These
generators stand in for them with the same shapes and value distributions (C-order, last axis
fastest, like the raw files ASZ reads):

* ``grf_field``: Gaussian random field with power spectrum P(k) ~ k^-alpha. It is FFT-filtered white
  noise with unit variance.
* ``c1_field``: 100x500x500, k^-11/3 GRF, 20 Gaussian blobs and white noise at 1e-4 of the range.
* ``c2_field``: 512^3, k^-5/3 GRF plus a tanh front of width 4 voxels on a random plane, with
  amplitude 10x the field's standard deviation.
* ``c3_fields``: 48 fields with dims U[96,512] and alpha U[3,5].
* ``c4_field``: 256^3 with per-octant anisotropic correlation lengths and slopes.
* ``c5_step``: a 1024x1024x512 time step (turbulence + front + zero slab), advected per step.

All generators take an explicit shape so tests can run the same recipe at small sizes.
"""
from __future__ import annotations

import numpy as np


def _kgrid(shape):
    ks = [np.fft.fftfreq(n) * n for n in shape[:-1]] + [np.fft.rfftfreq(shape[-1]) * shape[-1]]
    return np.meshgrid(*ks, indexing="ij", sparse=True)


def grf_field(shape, alpha, rng, aniso=(1.0, 1.0, 1.0)):
    """Unit-variance Gaussian random field with P(k) ~ |k|^-alpha (float64)."""
    shape = tuple(int(s) for s in shape)
    white = rng.standard_normal(shape)
    spec = np.fft.rfftn(white)
    k0, k1, k2 = _kgrid(shape)
    kk = np.sqrt((k0 * aniso[0]) ** 2 + (k1 * aniso[1]) ** 2 + (k2 * aniso[2]) ** 2)
    kk[0, 0, 0] = 1.0
    amp = kk ** (-alpha / 2.0)
    amp[0, 0, 0] = 0.0
    f = np.fft.irfftn(spec * amp, s=shape, axes=(0, 1, 2))
    f -= f.mean()
    sd = f.std()
    return f / sd if sd > 0 else f


def c1_field(seed=1, shape=(100, 500, 500), blobs=20):
    rng = np.random.default_rng(seed)
    f = grf_field(shape, 11.0 / 3.0, rng)
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij", sparse=True)
    for _ in range(blobs):
        c = [rng.uniform(0, n) for n in shape]
        s = rng.uniform(5, 40)
        a = rng.normal(0, 3)
        d2 = sum((g - ci) ** 2 for g, ci in zip(grids, c))
        f = f + a * np.exp(-d2 / (2 * s * s))
    rngv = float(f.max() - f.min())
    f = f + rng.standard_normal(shape) * (1e-4 * rngv)
    return f.astype(np.float32)


def _front(shape, rng, width=4.0):
    n = rng.standard_normal(3)
    n /= np.linalg.norm(n)
    c = [rng.uniform(0.25 * s, 0.75 * s) for s in shape]
    grids = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij", sparse=True)
    d = sum((g - ci) * ni for g, ci, ni in zip(grids, c, n))
    return np.tanh(d / width)


def c2_field(seed=2, shape=(512, 512, 512)):
    rng = np.random.default_rng(seed)
    f = grf_field(shape, 5.0 / 3.0, rng)
    f = f + 10.0 * f.std() * _front(shape, rng)
    return f.astype(np.float32)


def c3_fields(seed=3, count=48, lo=96, hi=512):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        shape = tuple(int(x) for x in rng.integers(lo, hi + 1, size=3))
        alpha = rng.uniform(3, 5)
        out.append(grf_field(shape, alpha, rng).astype(np.float32))
    return out


def c4_field(seed=4, shape=(256, 256, 256)):
    rng = np.random.default_rng(seed)
    f = np.empty(shape, dtype=np.float64)
    h = [s // 2 for s in shape]
    for o in range(8):
        sl = tuple(slice(0, h[a]) if not (o >> a) & 1 else slice(h[a], shape[a]) for a in range(3))
        sub = tuple(x.stop - x.start for x in sl)
        corr = rng.uniform(2, 64, size=3)
        slope = rng.uniform(2.5, 5)
        f[sl] = grf_field(sub, slope, rng, aniso=tuple(corr / corr.mean()))
    return f.astype(np.float32)


def c5_step(step, seed=5, shape=(1024, 1024, 512), velocity=(1.5, 0.7, 0.3)):
    """Time step `step`: step 0 advected by step*velocity with periodic trilinear resampling."""
    rng = np.random.default_rng(seed)
    f = grf_field(shape, 5.0 / 3.0, rng)
    f = f + 10.0 * f.std() * _front(shape, rng)
    z0 = int(rng.integers(0, shape[0] - shape[0] // 10))
    f[z0:z0 + shape[0] // 10] = 0.0
    if step:
        f = _advect(f, [v * step for v in velocity])
        f = f + rng.standard_normal(shape) * 1e-3 * float(f.max() - f.min())
    return f.astype(np.float32)


def _advect(f, shift):
    out = f
    for axis, s in enumerate(shift):
        i = int(np.floor(s))
        w = s - i
        a = np.roll(out, i, axis=axis)
        b = np.roll(out, i + 1, axis=axis)
        out = (1 - w) * a + w * b
    return out
