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
