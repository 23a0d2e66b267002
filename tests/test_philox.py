"""Philox4x32-10 restatement against the published known-answer vectors."""
import numpy as np

from oracle import philox as P


def test_philox_known_answers():
    # Random123 known-answer vectors for philox4x32-10
    cases = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in cases:
        got = P.philox4x32_10(*[np.array([c], np.uint32) for c in ctr], *key)
        assert tuple(int(g[0]) for g in got) == want


def test_thermal_gaussian_moments():
    xi = P.thermal_gaussians(200000, step=7, seed=123)
    assert abs(xi.mean()) < 0.01 and abs(xi.std() - 1.0) < 0.01
    assert not np.array_equal(xi, P.thermal_gaussians(200000, step=8, seed=123))


def _fma32(a, b, c):
    """fmaf on float32 operands: the exact product (48 bits fit a double) plus c,
    rounded to float32 (one double rounding of the sum, below the bound)."""
    return np.float32(np.float64(a) * np.float64(b) + np.float64(c))


def test_box_muller_series_branch():
    """The FP32 Box-Muller radius takes -ln u near u = 1 from the series
    v + v^2/2 + v^3/3 + v^4/4 in v = 1 - u, with v read from the complemented
    integer (exact, since v < 1/64 there).  In float32 arithmetic the series
    stays within 4 x 2^-24 relative of the exact -ln(1 - v) (measured 1.9 x
    2^-24) over the whole branch, down to the smallest v the 24-bit uniforms
    give (2^-25), and the complement is exact.  The far branch and the square
    root, sine and cosine run on the GPU's approximations and are checked there
    (tests/test_llg_gpu.py)."""
    k = np.concatenate([np.arange(2**24 - 4096, 2**24, dtype=np.uint64),
                        np.linspace(2**24 - 2**18, 2**24 - 4097, 4000).astype(np.uint64)])
    x = (k << np.uint64(8)).astype(np.uint32)
    u = ((x >> np.uint32(8)).astype(np.float64) + 0.5) / 2**24
    vc = ((~x >> np.uint32(8)).astype(np.float64) + 0.5) / 2**24
    v32 = vc.astype(np.float32)
    assert np.array_equal(v32.astype(np.float64), 1.0 - u)  # the complement is 1 - u exactly
    assert v32.max() < 1 / 64
    third = np.float32(1.0 / 3.0)
    p = np.array([_fma32(v, np.float32(0.25), third) for v in v32], np.float32)
    p = np.array([_fma32(v, q, np.float32(0.5)) for v, q in zip(v32, p)], np.float32)
    p = np.array([_fma32(v, q, np.float32(1.0)) for v, q in zip(v32, p)], np.float32)
    e = (v32 * p).astype(np.float64)
    exact = -np.log1p(-(1.0 - u))
    rel = np.abs(e - exact) / exact
    assert rel.max() < 4 * 2.0 ** -24, rel.max()
