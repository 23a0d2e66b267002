"""Higher-order anisotropy on the device (src/anisotropy/: fourth- and
sixth-order uniaxial, sixth-order cubic, rotated fourth-order cubic and Neel
surface anisotropy) against the reference's own fixtures
(tests/golden/sc6_aniso_ho.npz, fcc4_neel_rot.npz) and the FP64 oracle that
those fixtures pin.  The terms reach the device through
vgpu_set_anisotropy_ext."""
import numpy as np
import pytest

from conftest import load_golden, ref_spins

pytestmark = pytest.mark.gpu

CASES = [("sc6_aniso_ho", (1, 200)), ("fcc4_neel_rot", (1, 100))]


@pytest.mark.parametrize("name,steps", CASES)
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_fields_match_oracle(vgpu_lib, name, steps, prec):
    from oracle import oracle as O
    from vampire_b200 import vgpu
    s, _ = load_golden(name)
    with vgpu.Simulation(s, precision=prec) as sim:
        got = sim.fields()
    o = O.OracleSystem(s)
    want = o.spin_fields(s.spins) + o.external_fields(None)
    tol = 2e-6 if prec == "fp32" else 1e-12
    assert np.abs(got - want).max() <= tol * np.abs(want).max()


@pytest.mark.parametrize("name,steps", CASES)
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_trajectory_matches_reference(vgpu_lib, name, steps, prec):
    from vampire_b200 import vgpu
    s, d = load_golden(name)
    errs = {}
    with vgpu.Simulation(s, precision=prec) as sim:
        done = 0
        for t in steps:
            sim.llg_heun(t - done)
            done = t
            errs[t] = float(np.abs(sim.spins() - ref_spins(d, t)).max())
    print(f"{name} {prec}: {errs}")
    for t, e in errs.items():
        assert e <= (1e-12 if prec == "fp64" else 1e-5), (t, e)


@pytest.mark.parametrize("name,steps", CASES)
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_energies_match_reference(vgpu_lib, name, steps, prec):
    """Device energy statistics (anisotropy term now with every higher-order
    contribution) against the reference's energy_statistic_t output."""
    from vampire_b200 import vgpu
    s, d = load_golden(name)
    for t in (0, steps[-1]):
        with vgpu.Simulation(s, precision=prec) as sim:
            sim.set_spins(ref_spins(d, t))
            mid = sim.add_mask(*s.masks["system"])
            sim.stats_update(magnetization=True, energy=True)
            e, _, _ = sim.energy(mid)
        ref = d[f"energy_system_{t}"]
        rtol = 1e-11 if prec == "fp64" else 2e-6
        np.testing.assert_allclose(np.asarray(e).reshape(-1)[: ref.size], ref.reshape(-1), rtol=rtol,
                                   atol=rtol * np.abs(ref).max())


def test_extension_validation(vgpu_lib):
    from vampire_b200 import vgpu
    s, _ = load_golden("sc6_aniso_ho")
    with vgpu.Simulation(s) as sim:
        x, keep = vgpu._aniso_ext({**s.aniso, "u4": True, "ku4": None})
        assert vgpu.lib().vgpu_set_anisotropy_ext(sim.handle, vgpu.C.byref(x)) == vgpu.ERR_ARG
        bad = dict(s.aniso)
        bad["ku6"] = np.array([np.nan])
        x, keep = vgpu._aniso_ext(bad)
        assert vgpu.lib().vgpu_set_anisotropy_ext(sim.handle, vgpu.C.byref(x)) == vgpu.ERR_ARG
