"""Biquadratic exchange on the device (src/exchange/biquadratic_fields.cpp,
biquadratic_energy.cpp) against the reference's own fixtures
(tests/golden/sc6_biquadratic_t0.npz, _t300.npz) and the FP64 oracle that
they pin; the term reaches the device through vgpu_set_biquadratic."""
import numpy as np
import pytest

from conftest import load_golden, ref_spins

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_fields_match_oracle(vgpu_lib, prec):
    from oracle import oracle as O
    from vampire_b200 import vgpu
    s, _ = load_golden("sc6_biquadratic_t0")
    with vgpu.Simulation(s, precision=prec) as sim:
        got = sim.fields()
    o = O.OracleSystem(s)
    want = o.spin_fields(s.spins) + o.external_fields(None)
    tol = 2e-6 if prec == "fp32" else 1e-12
    assert np.abs(got - want).max() <= tol * np.abs(want).max()


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_trajectories_match_reference(vgpu_lib, prec, tol):
    from vampire_b200 import vgpu
    s, d = load_golden("sc6_biquadratic_t0")
    with vgpu.Simulation(s, precision=prec) as sim:
        sim.llg_heun(1)
        assert np.abs(sim.spins() - ref_spins(d, 1)).max() <= tol
        sim.llg_heun(199)
        assert np.abs(sim.spins() - ref_spins(d, 200)).max() <= tol
    s, d = load_golden("sc6_biquadratic_t300")
    with vgpu.Simulation(s, precision=prec) as sim:
        for t in (1, 2):
            sim.set_noise_replay(d[f"xi_{t}"])
            sim.llg_heun(1)
            assert np.abs(sim.spins() - ref_spins(d, t)).max() <= tol, t


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_exchange_energy_includes_biquadratic(vgpu_lib, prec):
    from vampire_b200 import vgpu
    s, d = load_golden("sc6_biquadratic_t0")
    for t in (0, 200):
        with vgpu.Simulation(s, precision=prec) as sim:
            sim.set_spins(ref_spins(d, t))
            mid = sim.add_mask(*s.masks["system"])
            sim.stats_update(magnetization=True, energy=True)
            e, _, _ = sim.energy(mid)
        want = d[f"energy_system_{t}"]
        tol = 2e-6 if prec == "fp32" else 1e-11
        assert np.abs(e - want).max() < tol * (np.abs(want).max() + 1.0)


def test_biquadratic_refused_where_unsupported(vgpu_lib):
    from vampire_b200 import vgpu
    s, _ = load_golden("sc6_biquadratic_t0")
    with vgpu.Simulation(s) as sim:
        with pytest.raises(vgpu.VGPUError):
            sim.set_owned(s.n // 2, 0)
