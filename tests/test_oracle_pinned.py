"""The FP64 CPU oracle (oracle/vref.c) against the reference program itself.

The golden fixtures were produced by the reference's own objects (see
tests/golden/make_golden.py); the oracle must reproduce them to FP64
rounding.  This pins the checker that the GPU tests use.
"""
import numpy as np
import pytest

from conftest import load_golden, ref_spins
from oracle import oracle as O


@pytest.mark.parametrize("steps", [1, 2, 10, 100, 1000, 2000])
def test_sc8_t0_trajectory(steps):
    s, d = load_golden("sc8_t0")
    o = O.OracleSystem(s)
    got = o.llg_heun(s.spins, steps)
    assert np.abs(got - ref_spins(d, steps)).max() < 1e-12


def test_sc20_t0_config0_trajectory():
    """Config-0 system, 10,000 deterministic steps: the oracle follows the
    reference step for step."""
    s, d = load_golden("sc20_t0")
    o = O.OracleSystem(s)
    got = s.spins
    for a, b in [(0, 1), (1, 100), (100, 10000)]:
        got = o.llg_heun(got, b - a)
        assert np.abs(got - ref_spins(d, b)).max() < 1e-12, b


@pytest.mark.parametrize("name,steps", [("sc10_t300", 2), ("sc6_open_t300", 3), ("fcc4_dmi_t300", 2)])
def test_replayed_noise_steps(name, steps):
    """T>0: with the reference's own Gaussian stream the oracle reproduces its
    stochastic Heun steps (thermal field sigma*sqrt(T)*xi, x|y|z blocks)."""
    s, d = load_golden(name)
    o = O.OracleSystem(s)
    got = s.spins
    for t in range(1, steps + 1):
        got = o.llg_heun(got, 1, xi=d[f"xi_{t}"])
        if f"sx_{t}" in d:
            assert np.abs(got - ref_spins(d, t)).max() < 1e-12, t


def test_fcc_dmi_t0_200_steps():
    s, d = load_golden("fcc4_dmi_t0")
    o = O.OracleSystem(s)
    got = o.llg_heun(s.spins, 200)
    assert np.abs(got - ref_spins(d, 200)).max() < 1e-11


def test_single_spin_known_answer():
    """The reference's own known-answer test (tests/physical/AppliedField,
    applied_field_errors.py): Sx = sech(l a) cos a, Sy = sech(l a) sin a,
    Sz = tanh(l a), a = gamma H t/(1+l^2); max error < 1e-6."""
    s, d = load_golden("single_spin_applied")
    o = O.OracleSystem(s)
    lam, H, g, dt = 1.0, 10.0, 1.76e11, 1e-16
    for t in (50, 1000, 5000, 10000):
        got = o.llg_heun(s.spins, t)[:, 0]
        assert np.abs(got - ref_spins(d, t)[:, 0]).max() < 1e-13
        arg = g * H * t * dt / (1 + lam * lam)
        exact = np.array([np.cos(arg) / np.cosh(lam * arg), np.sin(arg) / np.cosh(lam * arg), np.tanh(lam * arg)])
        assert np.abs(got - exact).max() < 1e-6


@pytest.mark.parametrize("name,step", [("sc20_t0", 10000), ("fcc4_dmi_t300", 2), ("sc6_open_t300", 3)])
def test_statistics(name, step):
    """Magnetisation and energy reductions (statistics/magnetization.cpp:134,
    statistics/energy.cpp:141) on the reference's own masks."""
    s, d = load_golden(name)
    o = O.OracleSystem(s)
    sp = ref_spins(d, step)
    mask, size = s.masks["system"]
    np.testing.assert_allclose(o.magnetization(sp, mask, size), d[f"mag_system_{step}"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(o.energy(sp, mask, size), d[f"energy_system_{step}"], rtol=1e-11, atol=1e-9)
    if f"mag_material_{step}" in d:
        mask, size = s.masks["material"]
        np.testing.assert_allclose(o.magnetization(sp, mask, size), d[f"mag_material_{step}"], rtol=1e-12,
                                   atol=1e-12)
        np.testing.assert_allclose(o.energy(sp, mask, size), d[f"energy_material_{step}"], rtol=1e-11, atol=1e-9)


def test_oracle_detects_a_planted_error():
    """A mistake planted in the oracle's inputs (one bond's coupling) must
    show up against the reference fixture: the checker is not vacuous."""
    s, d = load_golden("sc8_t0")
    bad = s.copy()
    bad.jlist = bad.jlist.copy()
    bad.jlist[7] *= 1.001
    got = O.OracleSystem(bad).llg_heun(bad.spins, 10)
    assert np.abs(got - ref_spins(d, 10)).max() > 1e-9


@pytest.mark.parametrize("name,steps", [("sc6_aniso_ho", (1, 200)), ("fcc4_neel_rot", (1, 100))])
def test_higher_order_anisotropy(name, steps):
    """Fourth/sixth-order uniaxial, sixth-order cubic, rotated cubic and Neel
    surface anisotropy (src/anisotropy/*.cpp): the oracle follows the
    reference trajectory and reproduces its anisotropy energies."""
    s, d = load_golden(name)
    assert s.aniso is not None
    o = O.OracleSystem(s)
    got = s.spins
    done = 0
    for t in steps:
        got = o.llg_heun(got, t - done)
        done = t
        assert np.abs(got - ref_spins(d, t)).max() < 1e-12, t
    for t in (0, steps[-1]):
        sp = ref_spins(d, t)
        mask, size = s.masks["system"]
        np.testing.assert_allclose(o.energy(sp, mask, size), d[f"energy_system_{t}"], rtol=1e-11, atol=1e-9)


def test_higher_order_anisotropy_pins_each_term():
    """Each higher-order term matters at the fixture's tolerance: dropping any
    one of them moves the 200-step trajectory off the reference."""
    s, d = load_golden("sc6_aniso_ho")
    for key in ("u4", "u6", "c6"):
        bad = s.copy()
        bad.aniso = dict(s.aniso)
        bad.aniso[key] = False
        got = O.OracleSystem(bad).llg_heun(bad.spins, 200)
        assert np.abs(got - ref_spins(d, 200)).max() > 1e-9, key


def _derived_from_rows(mag_rows, e_rows, sat, norm, T):
    """NumPy restatement of the reference's derived statistics
    (statistics/susceptibility.cpp, specific_heat.cpp, standard_deviation.cpp)
    from per-update magnetisation rows (m_x, m_y, m_z, |m|) and total energies."""
    m = np.asarray(mag_rows)
    cnt = len(m)
    mm = m[:, 3]
    s1 = np.stack([m[:, 0] * mm, m[:, 1] * mm, m[:, 2] * mm, mm], 1).sum(0)
    s2 = np.stack([m[:, 0] ** 2 * mm ** 2, m[:, 1] ** 2 * mm ** 2, m[:, 2] ** 2 * mm ** 2, mm ** 2], 1).sum(0)
    sus = 9.274e-24 / (1.3806503e-23 * T) * sat * (s2 / cnt - s1 ** 2 / cnt ** 2)
    E = np.asarray(e_rows)
    sh = 9.27400999e-24 / (1.3806503e-23 * T * T) / norm * ((E ** 2).sum() / len(E) - E.sum() ** 2 / len(E) ** 2)
    std = m.std(axis=0)
    return sus, sh, std


def test_derived_statistics():
    """The oracle's replayed trajectory, reduced every step, gives the
    reference's susceptibility, specific heat and standard deviation."""
    s, d = load_golden("sc6_derived_t600")
    o = O.OracleSystem(s)
    mask, size = s.masks["system"]
    sp = s.spins
    rows, es = [], []
    for t in range(0, 21):
        if t > 0:
            sp = o.llg_heun(sp, 1, xi=d[f"xi_{t}"])
        rows.append(o.magnetization(sp, mask, size)[:4])
        es.append(o.energy(sp, mask, size)[0])
    assert np.abs(sp - ref_spins(d, 20)).max() < 1e-12
    sat = float(s.mu_s_muB()[mask == 0].sum())
    sus, sh, std = _derived_from_rows(rows, es, sat, float(np.sum(mask == 0)), 600.0)
    np.testing.assert_allclose(sus, d["sus_system"], rtol=1e-9)
    np.testing.assert_allclose(sh, d["spec_heat_system"][0], rtol=1e-9)
    np.testing.assert_allclose(std, d["std_material"], rtol=1e-7)


def test_llg_midpoint_deterministic():
    """sim::LLG_Midpoint (src/simulate/LLGMidpoint.cpp): 100 T=0 steps."""
    s, d = load_golden("sc8_midpoint_t0")
    o = O.OracleSystem(s)
    got = o.llg_midpoint(s.spins, 1)
    assert np.abs(got - ref_spins(d, 1)).max() < 1e-13
    got = o.llg_midpoint(got, 99)
    assert np.abs(got - ref_spins(d, 100)).max() < 1e-12


def test_llg_midpoint_replayed_noise():
    s, d = load_golden("sc8_midpoint_t300")
    o = O.OracleSystem(s)
    got = s.spins
    for t in (1, 2):
        got = o.llg_midpoint(got, 1, xi=d[f"xi_{t}"])
        assert np.abs(got - ref_spins(d, t)).max() < 1e-12, t


def test_biquadratic_exchange():
    """Biquadratic exchange (src/exchange/biquadratic_fields.cpp,
    biquadratic_energy.cpp): 200 T=0 steps, replayed T>0 steps and the
    exchange energy including the biquadratic term, against the reference."""
    s, d = load_golden("sc6_biquadratic_t0")
    assert s.biquadratic is not None
    o = O.OracleSystem(s)
    got = o.llg_heun(s.spins, 1)
    assert np.abs(got - ref_spins(d, 1)).max() < 1e-13
    got = o.llg_heun(got, 199)
    assert np.abs(got - ref_spins(d, 200)).max() < 1e-12
    mask, size = s.masks["system"]
    for t in (0, 200):
        np.testing.assert_allclose(o.energy(ref_spins(d, t), mask, size), d[f"energy_system_{t}"], rtol=1e-11,
                                   atol=1e-9)
    s, d = load_golden("sc6_biquadratic_t300")
    o = O.OracleSystem(s)
    got = s.spins
    for t in (1, 2):
        got = o.llg_heun(got, 1, xi=d[f"xi_{t}"])
        assert np.abs(got - ref_spins(d, t)).max() < 1e-12, t
    bad = s.copy()
    bad.biquadratic = None
    assert np.abs(O.OracleSystem(bad).llg_heun(s.spins, 1, xi=d["xi_1"]) - ref_spins(d, 1)).max() > 1e-9


EXCH_FIXTURES = ["tet_iso_bond", "tet_vec_bond", "tet_ten_bond", "sc6_vec"]


@pytest.mark.parametrize("name", EXCH_FIXTURES)
def test_exchange_forms_trajectory_and_energy(name):
    """Per-bond isotropic, vectorial and tensorial exchange from a unit-cell
    file, and the normalised vectorial form (src/exchange/exchange_fields.cpp
    :49-163, exchange/energy.cpp): 200 T=0 steps and the energies at step
    200 follow the reference; one replayed-noise step at 300 K."""
    s, d = load_golden(f"{name}_t0")
    o = O.OracleSystem(s)
    got, done = s.spins, 0
    for t in (1, 100, 200):
        got = o.llg_heun(got, t - done)
        done = t
        assert np.abs(got - ref_spins(d, t)).max() < 1e-12, t
    mask, size = s.masks["system"]
    e = o.energy(ref_spins(d, 200), mask, size)
    want = d["energy_system_200"]
    assert np.abs(e - want).max() < 1e-11 * np.abs(want).max()
    s3, d3 = load_golden(f"{name}_t300")
    o3 = O.OracleSystem(s3)
    got = s3.spins
    for t in (1, 2):
        got = o3.llg_heun(got, 1, xi=d3[f"xi_{t}"])
        assert np.abs(got - ref_spins(d3, t)).max() < 1e-12, t


def test_cmc_restatement_keeps_the_constraint():
    """The restated constrained pair rule (cmc.cpp:282-490) in the
    reference's own frame (tests/golden/cmc_sc12.npz): accepted pair moves
    keep the moment perpendicular to the constraint, spins stay unit, and the
    running moment equals the spins' moment."""
    from conftest import GOLDEN
    d = dict(np.load(GOLDEN / "cmc_sc12.npz"))
    s = O.system_from_dump(d)
    s.params.temperature = 600.0
    P, pv = d["cmc_frame"][:9].reshape(3, 3), d["cmc_frame"][9:12]
    sp = np.tile(pv[:, None], (1, s.n))
    mu = s.mu_s_muB()
    M = (sp * mu).sum(1)
    o = O.OracleSystem(s)
    rng = np.random.default_rng(3)
    K = 200
    for _ in range(5):
        pairs = rng.permutation(s.n)[: 2 * K].reshape(K, 2)
        rnd = np.concatenate([rng.standard_normal(3 * K), rng.random(K)])
        sp, M2, cnt = o.cmc_pairs(sp, pairs, rnd, P, pv, M)
        assert cnt[0] > 0
        perp = lambda v: v - (v @ pv) * pv
        assert np.abs(perp(M2) - perp(M)).max() < 1e-10 * np.abs(M).max()
        assert np.abs(np.linalg.norm(sp, axis=0) - 1.0).max() < 1e-14
        assert np.abs((sp * mu).sum(1) - M2).max() < 1e-9 * np.abs(M2).max()
        M = M2
