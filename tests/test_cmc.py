"""Constrained Monte Carlo (montecarlo::cmc_step, src/montecarlo/cmc.cpp:
282-490) on the device against the reference.

* frame: the device's constraint rotation equals the reference's
  polar_rot_matrix output (tests/golden/cmc_sc12.npz, dumped by the harness);
* the pair rule: one phase of replayed pair moves (the same pairs and random
  numbers) equals the oracle's restatement of the reference's rule
  (oracle/vref.c vref_cmc_pairs): FP64 to 1e-12 with identical counters,
  FP32 with at most one decision flipped at the rounding threshold; the
  moment perpendicular to the constraint is kept;
* statistics: the device chain reproduces the reference's own chain on SC
  12^3 (phi = 30, theta = 45 degrees): <m . e> within 3.5 standard errors at
  400 K and 900 K, the perpendicular moment zero to rounding.
"""
import numpy as np
import pytest

from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu


def _phase_pairs(col, rng, K):
    """K disjoint pairs of atoms of one colour."""
    atoms = np.flatnonzero(col == 0)
    pick = rng.permutation(atoms)[: 2 * K]
    return pick.reshape(K, 2)


@pytest.mark.parametrize("name", ["sc10_t300", "fcc4_dmi_t300", "tet_ten_bond_t300"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_replayed_phase_matches_oracle(vgpu_lib, name, prec):
    from oracle import oracle as O
    from vampire_b200 import vgpu
    s, _ = load_golden(name)
    s.params.temperature = 500.0
    o = O.OracleSystem(s)
    rng = np.random.default_rng(8)
    with vgpu.Simulation(s, precision=prec) as sim:
        sim.cmc_setup(30.0, 45.0, init_spins=True)
        P, pv = sim.cmc_frame()
        col = sim.mc_colours()
        spins = sim.spins()
        M = (spins * s.mu_s_muB()).sum(axis=1)
        tot = np.zeros(3, dtype=np.int64)
        for phase in range(4):
            K = min(np.sum(col == 0) // 2, 40)
            pairs = _phase_pairs(col, rng, K)
            rnd = np.concatenate([rng.standard_normal(3 * K), rng.random(K)])
            sim.cmc_pairs(pairs, rnd, moment=M)
            want, M_o, cnt = o.cmc_pairs(spins, pairs, rnd, P, pv, M)
            got = sim.spins()
            Mg, _ = sim.cmc_state()
            diff = np.abs(got - want).max(axis=0)
            if prec == "fp64":
                assert diff.max() < 1e-12, diff.max()
                assert np.abs(Mg - M_o).max() < 1e-9
            else:
                assert np.sum(diff > 1e-5) <= 2  # one flipped pair moves two spins
            # the moment perpendicular to the constraint is kept by every move
            perp = M_o - (M_o @ pv) * pv
            assert np.abs(perp - (M - (M @ pv) * pv)).max() < 1e-9 * np.abs(M).max()
            spins, M = got, Mg
            tot += cnt
        assert tot[0] > 0 and tot[1] > 0


def test_frame_matches_reference(vgpu_lib):
    from oracle import oracle as O
    from vampire_b200 import vgpu
    d = dict(np.load(GOLDEN / "cmc_sc12.npz"))
    s = O.system_from_dump(d)
    with vgpu.Simulation(s) as sim:
        sim.cmc_setup(30.0, 45.0)
        P, pv = sim.cmc_frame()
    np.testing.assert_allclose(P.ravel(), d["cmc_frame"][:9], atol=1e-15)
    np.testing.assert_allclose(pv, d["cmc_frame"][9:12], atol=1e-15)


def _blocks(x, nb=10):
    b = x[: len(x) // nb * nb].reshape(nb, -1).mean(1)
    return x.mean(), b.std(ddof=1) / np.sqrt(nb)


@pytest.mark.parametrize("T", [400.0, 900.0])
def test_chain_matches_reference_statistically(vgpu_lib, T):
    from oracle import oracle as O
    from vampire_b200 import vgpu
    d = dict(np.load(GOLDEN / "cmc_sc12.npz"))
    s = O.system_from_dump(d)
    s.params.H_applied = 0.0
    s.params.temperature = T
    eq, av, every = (int(x) for x in d["sweeps"])
    pv = d["cmc_frame"][9:12]
    ref = d[f"m_trace_{int(T)}"] @ pv
    reps, pars, perps = 4, [], []
    for r in range(reps):
        with vgpu.Simulation(s, noise_seed=900 + r) as sim:
            sim.cmc_setup(30.0, 45.0, init_spins=True)
            msat = s.mu_s_muB().sum()
            sim.cmc_sweep(eq)
            tr = []
            for _ in range(av // every):
                sim.cmc_sweep(every)
                M, _ = sim.cmc_state()
                tr.append(M / msat)
            tr = np.array(tr)
            pars.append(tr @ pv)
            perps.append(np.abs(tr - np.outer(tr @ pv, pv)).max())
            _, cnt = sim.cmc_state()
            assert cnt[1] > 0 and cnt[1] + cnt[2] + cnt[3] == cnt[0]
    g = np.concatenate(pars)
    mg = g.mean()
    eg = np.std([p.mean() for p in pars], ddof=1) / np.sqrt(reps)
    mr, er = _blocks(ref)
    z = abs(mg - mr) / np.hypot(eg, er)
    print(f"T={T}: <m.e> gpu {mg:.5f} +- {eg:.5f}, reference {mr:.5f} +- {er:.5f}, z {z:.2f}; "
          f"max perpendicular {max(perps):.2e}")
    assert z <= 3.5
    assert max(perps) < 1e-5


def test_hybrid_frames_match_reference(vgpu_lib):
    from oracle import oracle as O
    from vampire_b200 import vgpu
    d = dict(np.load(GOLDEN / "cmc_hybrid_sc12.npz"))
    s = O.system_from_dump(d)
    fr = d["cmc_frames"].reshape(2, 12)
    with vgpu.Simulation(s) as sim:
        sim.cmc_setup_materials([1, 0], [30.0, 0.0], [45.0, 0.0])
        P, pv = sim.cmc_frame()
    np.testing.assert_allclose(P.ravel(), fr[0, :9], atol=1e-15)
    np.testing.assert_allclose(pv, fr[0, 9:], atol=1e-15)


def test_hybrid_chain_matches_reference_statistically(vgpu_lib):
    """Hybrid constrained Monte Carlo (montecarlo::cmc_mc_step): SC 12^3 A/B
    alloy at 500 K, A constrained along (30, 45) degrees, B free, against the
    reference's own chain (tests/golden/cmc_hybrid_sc12.npz): A's moment
    along its constraint and B's moment projected on it within 3.5 standard
    errors; A's moment perpendicular to the constraint zero to rounding."""
    from oracle import oracle as O
    from vampire_b200 import vgpu
    d = dict(np.load(GOLDEN / "cmc_hybrid_sc12.npz"))
    s = O.system_from_dump(d)
    s.params.H_applied = 0.0
    s.params.temperature = 500.0
    eq, av, every = (int(x) for x in d["sweeps"])
    pv = d["cmc_frames"].reshape(2, 12)[0, 9:]
    ref = d["mat_trace"].reshape(-1, 2, 3)
    chains_a, chains_b, perp = [], [], 0.0
    for seed in range(4):
        with vgpu.Simulation(s, noise_seed=300 + seed) as sim:
            sim.cmc_setup_materials([1, 0], [30.0, 0.0], [45.0, 0.0])
            mid = sim.add_mask(*s.masks["material"])
            sim.cmc_sweep(eq)
            a, b = [], []
            for _ in range(av // every):
                sim.cmc_sweep(every)
                sim.stats_update(magnetization=True)
                m, _, _ = sim.magnetization(mid)
                rows = np.asarray(m).reshape(-1, 4)[:2]
                vec = rows[:, :3] * rows[:, 3:4]
                a.append(vec[0] @ pv)
                b.append(vec[1] @ pv)
                perp = max(perp, float(np.abs(vec[0] - (vec[0] @ pv) * pv).max()))
            _, cnt = sim.cmc_state()
            assert cnt[1] > 0 and abs(cnt[1] + cnt[2] + cnt[3] - cnt[0]) < 0.5
        chains_a.append(np.mean(a))
        chains_b.append(np.mean(b))
    for name, g, r in (("A.e", chains_a, ref[:, 0, :] @ pv), ("B.e", chains_b, ref[:, 1, :] @ pv)):
        mg, eg = np.mean(g), np.std(g, ddof=1) / np.sqrt(len(g))
        mr, er = _blocks(r)
        z = abs(mg - mr) / np.hypot(eg, er)
        print(f"hybrid {name}: gpu {mg:.5f} +- {eg:.5f}, reference {mr:.5f} +- {er:.5f}, z {z:.2f}")
        assert z <= 3.5
    assert perp < 1e-5
