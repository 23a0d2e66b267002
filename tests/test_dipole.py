"""Macrocell dipole field (K5/K6) against the reference's own cell fields.

tests/golden/fcc10_dipole_{tensor,macrocell}.npz hold the reference's
cells::mag_array, dipole::cells_field_array and cells_mu0Hd_field_array at
start-up and after the update at step 100, and its T=0 trajectory across that
update.
"""
import numpy as np
import pytest

from conftest import load_golden, ref_spins


def _cells(d, s, solver):
    return {"atom_cell": d["cell_id"], "cell_pos_mom": d["cell_pos_mom"], "cell_volume": d["cell_volume"],
            "cell_natoms": d["cell_natoms"], "macro_cell_size": 7.08, "cutoff": 2.0, "update_rate": 100,
            "solver": solver, "coords": s.coords}


def _ref_cells(d, t):
    return (np.stack([d[f"cmag_{c}_{t}"] for c in "xyz"]), np.stack([d[f"cfield_{c}_{t}"] for c in "xyz"]),
            np.stack([d[f"chd_{c}_{t}"] for c in "xyz"]))


@pytest.mark.parametrize("solver", ["tensor", "macrocell"])
def test_restatement_matches_reference(solver):
    """The NumPy restatement reproduces the reference's cell fields."""
    from oracle import dipole_ref as D
    s, d = load_golden(f"fcc10_dipole_{solver}")
    nc = d["cell_natoms"].size
    mag = D.cell_moments(s.spins, s.materials["mu_s_SI"][s.type], d["cell_id"], nc)
    m0, b0, h0 = _ref_cells(d, 0)
    np.testing.assert_allclose(mag, m0, rtol=1e-12, atol=1e-36)
    T = D.tensors(d["cell_pos_mom"], d["cell_natoms"], 7.08, 2.0, solver, s.coords, d["cell_id"])
    B, H = D.cell_fields(mag, T, d["cell_natoms"], d["cell_volume"])
    assert np.abs(B - b0).max() < 1e-12 * np.abs(b0).max()
    assert np.abs(H - h0).max() < 1e-12 * np.abs(h0).max()


def test_oracle_llg_with_dipole_field_matches_reference():
    """The reference adds the cell B field to every atom of the cell
    (fields.cpp:291-316), refreshed after step 100."""
    from oracle import oracle as O
    s, d = load_golden("fcc10_dipole_tensor")
    _, b0, _ = _ref_cells(d, 0)
    _, b1, _ = _ref_cells(d, 100)
    cid = d["cell_id"]
    got = O.OracleSystem(s, dipole_field=b0[:, cid]).llg_heun(s.spins, 100)
    assert np.abs(got - ref_spins(d, 100)).max() < 1e-12
    got = O.OracleSystem(s, dipole_field=b1[:, cid]).llg_heun(got, 1)
    assert np.abs(got - ref_spins(d, 101)).max() < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["tensor", "macrocell"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("far", ["fft", "direct"])
def test_device_cell_fields(vgpu_lib, solver, prec, far):
    """Cell moments and fields against the reference's own cells.  The far
    field by FP64 FFT convolution (the golden cells sit on a regular grid)
    matches the reference's dense FP64 sum to 1e-12 in the FP64 build; the
    direct all-pairs sum of FP32 terms to 1e-5.  FP32 builds start from FP32
    spins (moments to 1e-6)."""
    from vampire_b200 import vgpu
    s, d = load_golden(f"fcc10_dipole_{solver}")
    with vgpu.Simulation(s, precision=prec) as sim:
        sim.set_option(vgpu.OPT_DIPOLE_FFT, 1 if far == "fft" else 0)
        sim.dipole_setup(_cells(d, s, solver))
        assert sim.dipole_method() == (vgpu.DIPOLE_FAR_FFT if far == "fft" else vgpu.DIPOLE_FAR_DIRECT)
        m, b, h = sim.dipole_cells()
    m0, b0, h0 = _ref_cells(d, 0)
    mtol = 1e-12 if prec == "fp64" else 1e-6
    assert np.abs(m - m0).max() < mtol * np.abs(m0).max()
    ftol = 1e-12 if (far == "fft" and prec == "fp64") else 1e-5
    assert np.abs(b - b0).max() < ftol * np.abs(b0).max()
    assert np.abs(h - h0).max() < ftol * np.abs(h0).max()


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(7, 5, 3), (1, 6, 2), (12, 1, 1)])
def test_fft_far_field_matches_direct_sum(vgpu_lib, shape):
    """Ragged grids (odd extents, single layers, a line of cells), random
    moments: the FFT far field equals the FP64 direct sum of the NumPy
    restatement, and the device all-pairs kernel to its FP32 tolerance."""
    from oracle import dipole_ref as D
    from vampire_b200 import system as S
    from vampire_b200 import vgpu
    nx, ny, nz = shape
    s = S.build("sc", nx * 2, ny * 2, nz * 2, 3.0, [S.Material(alpha=0.1, mu_s_muB=1.72)],
                np.array([[5e-21]]), S.SimParams(dt_SI=1e-16, temperature=0.0), spin_seed=5,
                periodic=(False, False, False))
    S.dipole_cells(s, size=6.0, atomic_volume=27.0, solver="macrocell", update_rate=0)
    out = {}
    for far in ("fft", "direct"):
        with vgpu.Simulation(s, precision="fp64") as sim:
            sim.set_option(vgpu.OPT_DIPOLE_FFT, 1 if far == "fft" else 0)
            sim.dipole_setup(s.cells)
            out[far] = sim.dipole_cells()
    c = s.cells
    nc = c["cell_natoms"].size
    mag = D.cell_moments(s.spins, s.materials["mu_s_SI"][s.type], c["atom_cell"], nc)
    T = D.tensors(c["cell_pos_mom"], c["cell_natoms"], c["macro_cell_size"], c["cutoff"], "macrocell", s.coords,
                  c["atom_cell"])
    B, H = D.cell_fields(mag, T, c["cell_natoms"], c["cell_volume"])
    scale = np.abs(B).max()
    assert np.abs(out["fft"][1] - B).max() < 1e-12 * scale
    assert np.abs(out["direct"][1] - B).max() < 1e-5 * scale
    assert np.abs(out["fft"][2] - H).max() < 1e-12 * np.abs(H).max()


@pytest.mark.gpu
def test_device_trajectory_across_dipole_update(vgpu_lib):
    """101 T=0 steps with the device dipole solver (update every 100 steps)
    follow the reference trajectory; the update at step 100 happens on the
    device with no host round trip."""
    from vampire_b200 import vgpu
    s, d = load_golden("fcc10_dipole_tensor")
    with vgpu.Simulation(s, precision="fp64") as sim:
        sim.dipole_setup(_cells(d, s, "tensor"))
        for t in (99, 100, 101):
            sim.llg_heun(t - sim.step)
            err = np.abs(sim.spins() - ref_spins(d, t)).max()
            assert err < 1e-8, (t, err)
            if t == 100:
                _, b, _ = sim.dipole_cells()
                _, b1, _ = _ref_cells(d, 100)
                assert np.abs(b - b1).max() < 1e-5 * np.abs(b1).max()


@pytest.mark.gpu
def test_host_dipole_field_path(vgpu_lib):
    """Hosts that keep the CPU dipole solver push per-atom fields
    (transfer_dipole_fields_from_cpu_to_gpu); the step uses them."""
    from vampire_b200 import vgpu
    s, d = load_golden("fcc10_dipole_tensor")
    _, b0, h0 = _ref_cells(d, 0)
    cid = d["cell_id"]
    with vgpu.Simulation(s, precision="fp64") as sim:
        sim.set_dipole_field(b0[:, cid], h0[:, cid])
        sim.llg_heun(100)
        assert np.abs(sim.spins() - ref_spins(d, 100)).max() < 1e-12
