"""Torque statistics against the reference's own stats::system_torque and
stats::max_torque (src/utility/statistics.cpp:221-325).

tests/golden/torque_*.npz hold, at T = 0, the reference's system torque,
per-material torque and max |S x H| for: an FCC 4^3 A/B alloy with tensor
exchange + three-site DMI + cubic anisotropy (steps 0 and 50), the per-bond
tensorial tetragonal cell (steps 0 and 50), and FCC 10^3 with the macrocell
dipole field (step 0).

* CPU: the oracle's total field (oracle/vref.c) with a NumPy cross product
  reproduces the reference's numbers (pins the checker);
* GPU: vgpu_torque_update / vgpu_torque_get through the C ABI, FP32 to 2e-6
  and FP64 to 1e-11 of the largest per-material component, the running
  means over repeated updates and the reset.
"""
import numpy as np
import pytest

from conftest import load_golden, ref_spins

CASES = [("torque_fcc4_t0", 0), ("torque_fcc4_t0", 50), ("torque_tet_t0", 0), ("torque_tet_t0", 50),
         ("torque_fcc10_dipole", 0)]


def _split(v, M):
    return v[:3], np.stack([v[3:3 + M], v[3 + M:3 + 2 * M], v[3 + 2 * M:3 + 3 * M]], axis=1), v[3 + 3 * M]


def _dipole_b(d):
    return np.stack([d[f"cfield_{c}_0"] for c in "xyz"])[:, d["cell_id"]]


@pytest.mark.parametrize("name,step", CASES)
def test_oracle_torque_matches_reference(name, step):
    from oracle import oracle as O
    s, d = load_golden(name)
    sp = ref_spins(d, step)
    o = O.OracleSystem(s, dipole_field=_dipole_b(d) if "cell_id" in d else None)
    H = o.spin_fields(sp) + o.external_fields(None)
    c = np.cross(sp.T, H.T).T
    mu = s.materials["mu_s_SI"][s.type]
    M = s.materials.size
    tot, mat, mx = _split(d[f"torque_{step}"], M)
    got_mat = np.stack([(c[:, s.type == m] * mu[s.type == m]).sum(1) for m in range(M)])
    scale = np.abs(mat).max()
    assert np.abs(got_mat - mat).max() < 1e-12 * scale
    assert np.abs(got_mat.sum(0) - tot).max() < 1e-12 * scale
    assert abs(np.linalg.norm(c, axis=0).max() - mx) < 1e-12 * mx


@pytest.mark.gpu
@pytest.mark.parametrize("name,step", CASES)
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_device_torque_matches_reference(vgpu_lib, name, step, prec):
    from vampire_b200 import vgpu
    s, d = load_golden(name)
    M = s.materials.size
    tot, mat, mx = _split(d[f"torque_{step}"], M)
    tol = 2e-6 if prec == "fp32" else 1e-11
    with vgpu.Simulation(s, precision=prec) as sim:
        if "cell_id" in d:
            sim.dipole_setup({"atom_cell": d["cell_id"], "cell_pos_mom": d["cell_pos_mom"],
                              "cell_volume": d["cell_volume"], "cell_natoms": d["cell_natoms"],
                              "macro_cell_size": 7.08, "cutoff": 2.0, "update_rate": 100, "solver": "macrocell",
                              "coords": s.coords})
        sim.set_spins(ref_spins(d, step))
        sim.torque_update()
        r = sim.torque()
        scale = np.abs(mat).max()
        assert r["count"] == 1
        assert np.abs(r["material"] - mat).max() < tol * scale, (r["material"], mat)
        assert np.abs(r["total"] - tot).max() < tol * scale
        assert abs(r["max"] - mx) < tol * mx
        # running means: two more updates of the same state
        sim.torque_update()
        sim.torque_update()
        r2 = sim.torque()
        assert r2["count"] == 3
        assert np.abs(r2["mean"] - r["total"]).max() < 1e-12 * scale
        assert np.abs(r2["material_mean"] - r["material"]).max() < 1e-12 * scale
        sim.stats_reset()
        r3 = sim.torque()
        assert r3["count"] == 0 and np.all(r3["mean"] == 0)
