"""The exchange forms the reference supports besides the benchmark's
tensor+DMI table, on the GPU against the reference's own trajectories.

* per-bond couplings read from a unit-cell file (the reference's
  non-normalised 'isotropic', 'vectorial' and 'tensorial' interaction types,
  src/exchange/unroll.cpp:52-105; fields exchange_fields.cpp:49-163): a
  two-material tetragonal cell whose couplings depend on the bond direction,
  so the library must hold them per bond (ISO_BOND, VEC_BOND, TENSOR_BOND);
* the normalised vectorial form from the material file's three-valued
  exchange-matrix (exchange_fields.cpp:82-117; VEC_TAB).

Tolerances as the other trajectory tests: FP32 1e-5, FP64 1e-12 per spin
component; energies 2e-6 (FP32) / 1e-11 (FP64) of the largest term.
"""
import numpy as np
import pytest

from conftest import load_golden, ref_spins

pytestmark = pytest.mark.gpu

CASES = [("tet_iso_bond", "iso_bond"), ("tet_vec_bond", "vec_bond"), ("tet_ten_bond", "tensor_bond"),
         ("sc6_vec", "vec_tab")]
TOL = {"fp32": 1e-5, "fp64": 1e-12}


@pytest.fixture(scope="module")
def V(vgpu_lib):
    from vampire_b200 import vgpu
    return vgpu


@pytest.mark.parametrize("name,fmt", CASES)
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_format_fields_and_t0_trajectory(V, name, fmt, prec):
    from oracle import oracle as O
    s, d = load_golden(f"{name}_t0")
    with V.Simulation(s, precision=prec) as sim:
        assert sim.exchange_format() == fmt
        got = sim.fields()
        o = O.OracleSystem(s)
        want = o.spin_fields(s.spins) + o.external_fields(None)
        assert np.abs(got - want).max() <= (2e-6 if prec == "fp32" else 1e-12) * np.abs(want).max()
        errs, done = {}, 0
        for t in (1, 100, 200):
            sim.llg_heun(t - done)
            done = t
            errs[t] = float(np.abs(sim.spins() - ref_spins(d, t)).max())
    print(f"{name} {prec} ({fmt}) error vs reference: {errs}")
    assert max(errs.values()) <= TOL[prec], errs


@pytest.mark.parametrize("name,fmt", CASES)
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_replayed_noise_steps(V, name, fmt, prec):
    s, d = load_golden(f"{name}_t300")
    with V.Simulation(s, precision=prec) as sim:
        assert sim.exchange_format() == fmt
        for t in (1, 2):
            sim.set_noise_replay(d[f"xi_{t}"])
            sim.llg_heun(1)
            err = float(np.abs(sim.spins() - ref_spins(d, t)).max())
            assert err <= TOL[prec], (t, err)


@pytest.mark.parametrize("name,fmt", CASES)
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_energies_match_reference(V, name, fmt, prec):
    s, d = load_golden(f"{name}_t0")
    with V.Simulation(s, precision=prec) as sim:
        sim.set_spins(ref_spins(d, 200))
        mid = sim.add_mask(*s.masks["system"])
        sim.stats_update(magnetization=True, energy=True)
        m, _, _ = sim.magnetization(mid)
        e, _, _ = sim.energy(mid)
    want_m, want_e = d["mag_system_200"], d["energy_system_200"]
    tol = 2e-6 if prec == "fp32" else 1e-11
    assert np.abs(m - want_m).max() < tol
    assert np.abs(e - want_e).max() < tol * (np.abs(want_e).max() + 1.0), (e, want_e)


@pytest.mark.parametrize("name", ["tet_ten_bond", "tet_vec_bond", "sc6_vec"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_replayed_mc_sweep(V, name, prec):
    """Monte Carlo energies with these exchange forms: three colour-ordered
    sweeps with replayed random numbers equal the oracle's restatement of
    the reference acceptance rule."""
    from oracle import oracle as O
    s, _ = load_golden(f"{name}_t300")
    s.params.temperature = 300.0
    rng = np.random.default_rng(5)
    o = O.OracleSystem(s)
    with V.Simulation(s, precision=prec) as sim:
        sim.mc_setup()
        col = sim.mc_colours()
        spins = s.spins.copy()
        for _ in range(3):
            rnd = np.concatenate([rng.standard_normal(3 * s.n), rng.random(s.n)])
            sim.mc_set_replay(rnd)
            sim.mc_sweep(1)
            spins, _ = o.mc_colour_sweep(spins, col, rnd)
            got = sim.spins()
            diff = np.abs(got - spins).max(axis=0)
            if prec == "fp64":
                assert diff.max() < 1e-12
            else:
                assert np.sum(diff > 1e-5) <= 1
                spins = got
