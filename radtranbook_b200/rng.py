"""Philox-4x32-10 on the host (NumPy), for seeded problem set-up: per-instance keys and
parameters of a batch, Gaussian random fields.  The same generator as the device one
(Salmon et al., SC'11), so host and device streams can be compared."""
from __future__ import annotations

import numpy as np


def philox4x32_10(ctr: np.ndarray, key: int) -> np.ndarray:
    """Philox-4x32-10 of counters ctr[(n, 4) uint32] under a 64-bit key (vectorised)."""
    c = np.asarray(ctr, dtype=np.uint64).reshape(-1, 4).copy()
    k0, k1 = np.uint64(key & 0xFFFFFFFF), np.uint64((key >> 32) & 0xFFFFFFFF)
    m32 = np.uint64(0xFFFFFFFF)
    M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
    for r in range(10):
        if r:
            k0 = (k0 + np.uint64(0x9E3779B9)) & m32
            k1 = (k1 + np.uint64(0xBB67AE85)) & m32
        p0 = M0 * c[:, 0]
        p1 = M1 * c[:, 2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & m32
        hi1, lo1 = p1 >> np.uint64(32), p1 & m32
        c = np.stack([hi1 ^ c[:, 1] ^ k0, lo1, hi0 ^ c[:, 3] ^ k1, lo0], axis=1)
    return c.astype(np.uint32)


def u01(x: np.ndarray) -> np.ndarray:
    """The device's 23-bit open-interval uniform, (2k+1) 2^-24."""
    return (((x.astype(np.uint64) >> np.uint64(9)) << np.uint64(1)) | np.uint64(1)).astype(np.float64) * 2.0 ** -24


def normals(n: int, key: int, tag: int) -> np.ndarray:
    """n standard normals (Box-Muller on Philox uniforms, counter (i, 0, 0, tag))."""
    m = (n + 1) // 2
    i = np.arange(m, dtype=np.uint64)
    z = np.zeros(m, dtype=np.uint64)
    u = u01(philox4x32_10(np.stack([i, z, z, z + np.uint64(tag)], 1), key))
    r = np.sqrt(-2.0 * np.log(u[:, 0]))
    a = 2.0 * np.pi * u[:, 1]
    return np.stack([r * np.cos(a), r * np.sin(a)], 1).reshape(-1)[:n]
