"""Synthetic-system builders against the reference's own construction."""
import numpy as np

from conftest import load_golden
from vampire_b200 import system as S


def _ref_bond_vectors(s, box):
    cnt = s.nl_end - s.nl_start + 1
    ai = np.repeat(np.arange(s.n), cnt)
    v = (s.coords[:, s.nl] - s.coords[:, ai]).T
    return v - box * np.round(v / box)


def test_dmi_tensors_match_reference():
    """The three-site DMI (dmi.cpp:46-221) rebuilt from the reference's own
    neighbour list, materials and positions equals its t_exchange_list."""
    s, d = load_golden("fcc4_dmi_t300")
    v = _ref_bond_vectors(s, 4 * 3.54)
    mats = S.derive_materials([S.Material(alpha=0.05, mu_s_muB=1.72, Kc=1e-24)] * 2, 1e-16)
    J = np.array([[11.2e-21, 5e-21], [5e-21, 11.2e-21]])
    jl = S.exchange_lists(s.nl_start, s.nl_end, s.nl, s.type, mats, J, S.EXCH_TENSORIAL)
    jl = S.add_dmi(jl, s.nl_start, s.nl_end, s.nl, v, s.type, mats, 0.1 * J)
    assert np.abs(jl - s.jlist).max() < 1e-12 * np.abs(s.jlist).max()


def test_uniform_fast_path_equals_generic():
    """The per-slot-pair fast path for periodic lattices gives the same
    tensors as the generic masked construction."""
    f = S.config_fcc_tensor(L=3, seed=7)
    coords, st, en, nl, vec = S.lattice("fcc", 3, 3, 3, 3.54)
    J = np.array([[11.2e-21, 5e-21], [5e-21, 11.2e-21]])
    base = S.exchange_lists(st, en, nl, f.type, f.materials, J, S.EXCH_TENSORIAL)
    fast = S.add_dmi(base, st, en, nl, vec, f.type, f.materials, 0.1 * J)
    # force the generic path by breaking row regularity (append an empty atom)
    st2 = np.append(st, st[-1]); en2 = np.append(en, st[-1] - 1)
    ty2 = np.append(f.type, 0).astype(np.int32)
    slow = S.add_dmi(base, st2, en2, nl, vec, ty2, f.materials, 0.1 * J)
    assert np.abs(fast - slow).max() < 1e-12 * np.abs(fast).max()
    assert np.abs(fast.reshape(-1, 3, 3)[:, 0, 1]).max() > 1.0  # DMI is present


def test_sc_neighbours_match_reference():
    """SC 20^3 periodic nearest-neighbour pairs equal the reference's CSR
    (as position pairs; atom numbering may differ)."""
    s, _ = load_golden("sc20_t0")
    mine = S.config_sc_llg(20)
    def pairs(sys_, a=3.0, L=20):
        cnt = sys_.nl_end - sys_.nl_start + 1
        ai = np.repeat(np.arange(sys_.n), cnt)
        p = np.round(sys_.coords / a).astype(int) % L
        key = lambda i: p[0, i] + L * (p[1, i] + L * p[2, i])
        return set(zip(key(ai).tolist(), key(sys_.nl).tolist()))
    assert pairs(s) == pairs(mine)
    assert np.allclose(mine.jlist, s.jlist[0])
    np.testing.assert_allclose(mine.materials[0]["ku2"], s.materials[0]["ku2"], rtol=1e-15)
    np.testing.assert_allclose(mine.materials[0]["H_th_sigma"], s.materials[0]["H_th_sigma"], rtol=1e-15)
    np.testing.assert_allclose(mine.materials[0]["one_oneplusalpha_sq"], s.materials[0]["one_oneplusalpha_sq"])


def test_temperature_replicas_are_disjoint_copies():
    from vampire_b200 import system as S
    base = S.config_sc_llg(4, temperature=0.0)
    Ts = [0.0, 300.0, 900.0]
    r = S.replicas(base, Ts)
    n, k = base.n, len(Ts)
    assert r.n == k * n and r.num_bonds == k * base.num_bonds
    assert r.params.local_temperature and not base.params.local_temperature
    for c in range(k):
        lo, hi = c * n, (c + 1) * n
        nl = r.nl[r.nl_start[lo]:r.nl_end[hi - 1] + 1]
        assert nl.min() >= lo and nl.max() < hi                     # no bond leaves its copy
        assert np.array_equal(nl - lo, base.nl)
        assert np.all(r.type[lo:hi] == base.type + c * base.num_materials)
        assert np.all(r.materials["temperature"][r.type[lo:hi]] == Ts[c])
        assert np.all(r.masks["replica"][0][lo:hi] == c)
    np.testing.assert_array_equal(r.spins[:, n:2 * n], base.spins)
