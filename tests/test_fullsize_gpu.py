"""Size-independent properties at the benchmark size: FCC 100^3 = 4,000,000
spins, tensor exchange + 3-site DMI, two materials, cubic anisotropy (the
workload bench.py times).  The oracle cannot follow 4M spins in test time, so
these check what holds at any size: the staged and plain passes agree bit for
bit (with the dipole field on), FP32 follows the FP64 build of the same
kernels, spins stay on the unit sphere, and at T = 0 the damped dynamics
lowers the energy step by step."""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fcc100():
    from vampire_b200 import system as S
    return S.config_fcc_tensor(L=100, seed=2024, temperature=300.0)


def test_staged_equals_plain_with_dipole(vgpu_lib, fcc100):
    """Plain and staged passes with 16-byte and compact bond records (the
    default here; 96 dictionary entries: material pair x bond vector), and
    the window-staged passes, agree bit for bit at 4M spins."""
    from vampire_b200 import system as S
    from vampire_b200 import vgpu as V
    s = copy.copy(fcc100)
    S.dipole_cells(s, size=2 * 3.54, atomic_volume=3.54 ** 3 / 4.0, solver="tensor", update_rate=100)
    out = {}
    for staged, compact, window, layout in ((0, 0, 0, V.RECORDS_WIDE), (0, 1, 0, V.RECORDS_COMPACT),
                                            (1, 0, 0, V.RECORDS_WIDE), (1, 1, 0, V.RECORDS_COMPACT),
                                            (1, 1, 1, V.RECORDS_WINDOW)):
        with V.Simulation(s, noise_seed=5) as sim:
            sim.set_option(V.OPT_STAGED_RECORDS, staged)
            sim.set_option(V.OPT_COMPACT_RECORDS, compact)
            sim.set_option(V.OPT_WINDOW_STAGING, window)
            sim.set_option(V.OPT_STAGE_BUFFERS, 1 if window else -1)
            lay, nd = sim.record_layout()
            assert lay == layout and 0 < nd <= 512
            sim.dipole_setup(s.cells)
            assert sim.dipole_method() == V.DIPOLE_FAR_FFT
            sim.llg_heun(3)
            out[staged, compact, window] = sim.spins()
    ref = out[0, 0, 0]
    for k, v in out.items():
        np.testing.assert_array_equal(ref, v, err_msg=str(k))
    assert np.abs(np.linalg.norm(ref, axis=0) - 1.0).max() < 1e-6


def test_fp32_follows_fp64_and_energy_decreases(vgpu_lib, fcc100):
    from vampire_b200 import vgpu as V
    s = copy.copy(fcc100)
    s.params = copy.copy(fcc100.params)
    s.params.temperature = 0.0
    spins = {}
    energies = []
    for prec in ("fp64", "fp32"):
        with V.Simulation(s, precision=prec) as sim:
            mid = sim.add_mask(*s.masks["system"])
            for _ in range(5):
                if prec == "fp64":
                    sim.stats_update(magnetization=False, energy=True)
                    e, _, _ = sim.energy(mid)
                    energies.append(e[0])
                sim.llg_heun(1)
            spins[prec] = sim.spins()
    assert np.abs(spins["fp32"] - spins["fp64"]).max() < 1e-5
    assert np.abs(np.linalg.norm(spins["fp64"], axis=0) - 1.0).max() < 1e-12
    # T = 0, alpha > 0, static fields: the total energy does not rise
    e = np.array(energies)
    assert np.all(np.diff(e) <= 1e-9 * np.abs(e).max()), e
