"""Device magnetisation and energy reductions (K4) against the reference's
own statistics (computed by the reference objects on the same spins)."""
import numpy as np
import pytest

from conftest import load_golden, ref_spins

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,step", [("sc20_t0", 10000), ("fcc4_dmi_t300", 2), ("sc6_open_t300", 3)])
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_stats_match_reference(vgpu_lib, name, step, prec):
    from vampire_b200 import vgpu
    s, d = load_golden(name)
    sp = ref_spins(d, step)
    with vgpu.Simulation(s, precision=prec) as sim:
        sim.set_spins(sp)
        ids = {k: sim.add_mask(*s.masks[k]) for k in ("system", "material")}
        sim.stats_update(magnetization=True, energy=True)
        sim.stats_update(magnetization=True, energy=True)
        for k, mid in ids.items():
            m, mean, cnt = sim.magnetization(mid)
            e, emean, ecnt = sim.energy(mid)
            assert cnt == 2 and ecnt == 2
            if f"mag_{k}_{step}" in d:
                want = d[f"mag_{k}_{step}"]
                tol = 2e-6 if prec == "fp32" else 1e-12
                assert np.abs(m - want).max() < tol
                assert np.abs(mean - 2 * want).max() < 2 * tol
            if f"energy_{k}_{step}" in d:
                want = d[f"energy_{k}_{step}"]
                scale = np.abs(want).max() + 1.0
                tol = 2e-6 if prec == "fp32" else 1e-11
                assert np.abs(e - want).max() < tol * scale, (e, want)
        sim.stats_reset()
        _, mean, cnt = sim.magnetization(ids["system"])
        assert cnt == 0 and np.all(mean == 0)


def test_stats_at_scale_checksum(vgpu_lib):
    """4M-spin FCC system: device reduction equals a float64 NumPy reduction
    of the downloaded spins (size-independent property)."""
    from vampire_b200 import system as S
    from vampire_b200 import vgpu
    s = S.config_fcc_tensor(L=60)
    with vgpu.Simulation(s) as sim:
        sim.llg_heun(5)
        sp = sim.spins()
        mid = sim.add_mask(*s.masks["material"])
        sim.stats_update()
        m, _, _ = sim.magnetization(mid)
    mu = s.mu_s_muB()
    for b in range(2):
        sel = s.type == b
        v = (sp[:, sel] * mu[sel]).sum(1)
        want = np.r_[v / np.linalg.norm(v), np.linalg.norm(v) / mu[sel].sum()]
        assert np.abs(m[4 * b:4 * b + 4] - want).max() < 1e-9


@pytest.mark.parametrize("prec,rtol", [("fp64", 1e-9), ("fp32", 1e-3)])
def test_derived_statistics_match_reference(vgpu_lib, prec, rtol):
    """Susceptibility, specific heat and standard deviation accumulated on the
    device over the reference's own 20 stochastic steps (replayed noise, one
    statistics update per step plus the initial one) against the values the
    reference's output functions print (tests/golden/sc6_derived_t600.npz)."""
    from vampire_b200 import vgpu
    s, d = load_golden("sc6_derived_t600")
    with vgpu.Simulation(s, precision=prec) as sim:
        mid = sim.add_mask(*s.masks["system"])
        sim.stats_update(magnetization=True, energy=True)
        for t in range(1, 21):
            sim.set_noise_replay(d[f"xi_{t}"])
            sim.llg_heun(1)
            sim.stats_update(magnetization=True, energy=True)
        sus, sh, sd = sim.stats_derived(mid, 600.0)
        sim.stats_reset()
        sus0, _, _ = sim.stats_derived(mid, 600.0)
    np.testing.assert_allclose(sus[0], d["sus_system"], rtol=rtol)
    np.testing.assert_allclose(sh[0], d["spec_heat_system"][0], rtol=rtol)
    np.testing.assert_allclose(sd[0], d["std_material"], rtol=rtol)
    assert not np.isfinite(sus0).all() or np.all(sus0 == 0)   # reset: no updates left


@pytest.mark.parametrize("name,step", [("fcc4_dmi_t300", 2), ("sc6_open_t300", 3)])
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_magnetization_only_path(vgpu_lib, name, step, prec):
    """The magnetisation-only reduction of small masks (register sums per
    thread) gives the reference's magnetisation like the full pass."""
    from vampire_b200 import vgpu
    s, d = load_golden(name)
    with vgpu.Simulation(s, precision=prec) as sim:
        sim.set_spins(ref_spins(d, step))
        for k in ("system", "material"):
            mid = sim.add_mask(*s.masks[k])
            sim.stats_update(magnetization=True, energy=False)
            m, _, cnt = sim.magnetization(mid)
            if f"mag_{k}_{step}" in d:
                tol = 2e-6 if prec == "fp32" else 1e-12
                assert np.abs(m - d[f"mag_{k}_{step}"]).max() < tol


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_copy_rows_pinned_and_pageable(vgpu_lib, prec):
    """vgpu_stats_copy_rows gives the same rows into pinned host memory (a
    kernel writes them through the device mapping) and into pageable memory
    (a copy), equal to the finalised rows vgpu_stats_get_magnetization reads,
    and ordered on the handle's stream: rows of consecutive steps, read after
    an event recorded behind each copy, follow the step's own update."""
    import torch
    from vampire_b200 import vgpu
    s, d = load_golden("fcc4_dmi_t300")
    s.params.temperature = 300.0
    with vgpu.Simulation(s, precision=prec, noise_seed=5) as sim:
        mid = sim.add_mask(*s.masks["material"])
        nb = s.masks["material"][1]
        pinned = [torch.zeros(9 * nb, dtype=torch.float64).pin_memory() for _ in range(2)]
        stream = torch.cuda.ExternalStream(sim.stream_ptr())
        for t in range(4):
            sim.llg_heun(1)
            sim.stats_update(magnetization=True)
            sim.stats_copy_rows(mid, pinned[t % 2].data_ptr())
            ev = torch.cuda.Event()
            ev.record(stream)
            ev.synchronize()
            m, _, _ = sim.magnetization(mid)
            got = pinned[t % 2].numpy().reshape(nb, 9)[:, :4]
            assert np.array_equal(got, m.reshape(nb, 4))
        pageable = np.zeros(9 * nb)
        sim.stats_copy_rows(mid, pageable.ctypes.data)
        sim.synchronize()
        assert np.array_equal(pageable, pinned[3 % 2].numpy())
