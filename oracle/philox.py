"""NumPy restatement of Philox4x32-10 and the Box-Muller transform.

TEST INFRASTRUCTURE ONLY: an independent check of the counter-based noise the
CUDA kernels generate in-register (vampire_b200/csrc/philox.cuh).  Follows the
published description (Salmon et al., SC'11): two 32x32->64 multiplies per
round with multipliers 0xD2511F53 and 0xCD9E8D57 and Weyl key increments
0x9E3779B9, 0xBB67AE85, ten rounds.
"""
import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint32).copy() for x in (c0, c1, c2, c3))
    k0 = np.uint32(k0)
    k1 = np.uint32(k1)
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = M0 * c0.astype(np.uint64)
            p1 = M1 * c2.astype(np.uint64)
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & MASK).astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & MASK).astype(np.uint32)
            c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
            k0 = np.uint32(k0 + W0)
            k1 = np.uint32(k1 + W1)
    return c0, c1, c2, c3


def thermal_gaussians(n: int, step: int, seed: int = 0, fp64: bool = False) -> np.ndarray:
    """The 3n thermal Gaussians (x|y|z blocks) of `step`: counter
    (atom, step_lo, step_hi, 0), key (seed_lo, seed_hi)."""
    i = np.arange(n, dtype=np.uint32)
    r = philox4x32_10(i, np.full(n, step & 0xFFFFFFFF, np.uint32), np.full(n, step >> 32, np.uint32),
                      np.zeros(n, np.uint32), seed & 0xFFFFFFFF, seed >> 32)
    if fp64:
        u = [(x.astype(np.float64) + 0.5) / 4294967296.0 for x in r]
    else:
        u = [((x >> np.uint32(8)).astype(np.float64) + 0.5) / 16777216.0 for x in r]
    r1 = np.sqrt(-2.0 * np.log(u[0]))
    r2 = np.sqrt(-2.0 * np.log(u[2]))
    gx = r1 * np.cos(2 * np.pi * u[1])
    gy = r1 * np.sin(2 * np.pi * u[1])
    gz = r2 * np.cos(2 * np.pi * u[3])
    return np.concatenate([gx, gy, gz])
