"""CPU oracle for the model-error field (test infrastructure only).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import
it.  It restates, in NumPy, the generator that ``go_grf_perturb`` /
``go_batch_grf_perturb`` (gpu-ocean_b200/csrc/model_error.cu) run on the GPU:

* Philox4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as
  easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64-bit multiplies by
  0xD2511F53 and 0xCD9E8D57, the high halves xored with the other counter
  words and the key, the key bumped by 0x9E3779B9 / 0xBB67AE85 per round;
* Box-Muller normals from 23-bit uniforms u = (2 floor(x / 2^9) + 1) / 2^24;
* a separable Gaussian filter exp(-d^2 / (2 s^2)), s = L / sqrt(2),
  R = ceil(3 s), normalised to unit sum of squares, periodic in x, over a
  noise grid ny + 2R rows high (rows wrap when north/south are periodic).

The reference gpu-ocean has no counterpart (its OceanStateNoise,
gpu_ocean/SWESimulators/OceanStateNoise.py, draws model error differently),
so this twin is pinned by its own known properties (unit variance, zero
mean, the Gaussian correlation) and compared with the GPU field in the GPU
tests.
"""

import math

import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 on arrays of 32-bit counter words (held in uint64)."""
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint64) & np.uint64(MASK) for x in (c0, c1, c2, c3))
    k0, k1 = np.uint64(k0 & MASK), np.uint64(k1 & MASK)
    m0, m1, mask = np.uint64(M0), np.uint64(M1), np.uint64(MASK)
    s32 = np.uint64(32)
    for _ in range(10):
        p0 = m0 * c0
        p1 = m1 * c2
        hi0, lo0 = p0 >> s32, p0 & mask
        hi1, lo1 = p1 >> s32, p1 & mask
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & mask, lo1, (hi0 ^ c3 ^ k1) & mask, lo0
        k0 = (k0 + np.uint64(W0)) & mask
        k1 = (k1 + np.uint64(W1)) & mask
    return c0, c1, c2, c3


def unit_open(x):
    return (2.0 * (np.asarray(x, dtype=np.uint64) >> np.uint64(9)).astype(np.float64) + 1.0) * 2.0 ** -24


def normals(l, event, key0, key1):
    """Normal numbers at linear indices l of the noise grid (float64)."""
    l = np.asarray(l, dtype=np.uint64)
    g = l >> np.uint64(2)
    lane = (l & np.uint64(3)).astype(np.int64)
    r0, r1, r2, r3 = philox4x32_10(g, np.full_like(g, event), np.zeros_like(g), np.zeros_like(g), key0, key1)
    a = np.where(lane < 2, r0, r2)
    b = np.where(lane < 2, r1, r3)
    rad = np.sqrt(-2.0 * np.log(unit_open(a)))
    ang = 2.0 * math.pi * unit_open(b)
    return np.where(lane & 1, rad * np.sin(ang), rad * np.cos(ang))


def filter_weights(corr_cells):
    s = float(corr_cells) / math.sqrt(2.0)
    R = int(math.ceil(3.0 * s))
    d = np.arange(-R, R + 1, dtype=np.float64)
    w = np.exp(-d * d / (2.0 * s * s))
    return w / np.sqrt(np.sum(w * w)), R


def field(nx, ny, key0, key1, event, corr_cells, periodic_y=False):
    """The unit-variance field (ny x nx, float64) the GPU adds (times std)."""
    w, R = filter_weights(corr_cells)
    yext = np.arange(ny + 2 * R)
    grow = R + np.mod(yext - R, ny) if periodic_y else yext
    x = np.arange(nx)
    l = (grow[:, None].astype(np.uint64) * np.uint64(nx) + x[None, :].astype(np.uint64))
    z = normals(l, event, key0, key1)                       # (ny + 2R) x nx
    zx = np.zeros_like(z)
    for k, wk in enumerate(w):
        zx += wk * np.roll(z, -(k - R), axis=1)             # periodic in x
    out = np.zeros((ny, nx))
    for k, wk in enumerate(w):
        out += wk * zx[k:k + ny]
    return out
