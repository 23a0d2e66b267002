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
    from vampire_b200 import system as S
    from vampire_b200 import vgpu as V
    s = copy.copy(fcc100)
    S.dipole_cells(s, size=2 * 3.54, atomic_volume=3.54 ** 3 / 4.0, solver="tensor", update_rate=100)
    out = {}
    for staged in (0, 1):
        with V.Simulation(s, noise_seed=5) as sim:
            sim.set_option(V.OPT_STAGED_RECORDS, staged)
            sim.dipole_setup(s.cells)
            assert sim.dipole_method() == V.DIPOLE_FAR_FFT
            sim.llg_heun(3)
            out[staged] = sim.spins()
    np.testing.assert_array_equal(out[0], out[1])
    assert np.abs(np.linalg.norm(out[1], axis=0) - 1.0).max() < 1e-6


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
