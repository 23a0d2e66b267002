"""Shards of one system on the GPU, through the C ABI.

Each rank's shard is its own handle (owned atoms then halo atoms,
vgpu_set_owned); here all shards share one GPU and the host moves the halo
blocks between the passes with vgpu_halo_pack / vgpu_halo_unpack and stream
synchronisation -- no kernel waits on another.  Owned spins must equal the
whole system stepped on one handle bit for bit (same bond order, same Philox
counters through noise_base), and the shards' raw statistics sums must add
up to the whole system's magnetisation.
"""
import os

import numpy as np
import pytest

from vampire_b200 import shard as SH
from vampire_b200 import system as S

pytestmark = pytest.mark.gpu


def _refresher(torch, plans, sims, dtype):
    """Host-driven halo refresh of every shard (pack, synchronise, unpack)."""
    idx = [{q: torch.as_tensor(ix, dtype=torch.int32, device="cuda") for q, ix in p.send.items()} for p in plans]

    def refresh(which):
        for sim in sims:
            sim.synchronize()
        bufs = {}
        for r, p in enumerate(plans):
            for q, ix in idx[r].items():
                out = torch.empty(3 * ix.numel(), dtype=dtype, device="cuda")
                sims[r].halo_pack(which, ix.data_ptr(), ix.numel(), out.data_ptr())
                bufs[(r, q)] = out
        for sim in sims:
            sim.synchronize()
        for r, p in enumerate(plans):
            for src, (first, count) in p.recv.items():
                sims[r].halo_unpack(which, first, count, bufs[(src, r)].data_ptr())
        for sim in sims:
            sim.synchronize()

    return refresh


def _step_shards(V, torch, plans, sims, steps, dtype):
    refresh = _refresher(torch, plans, sims, dtype)
    for _ in range(steps):
        for sim in sims:
            sim.llg_pass(V.PASS_PREDICTOR)
        refresh(V.STATE_PREDICTOR)
        for sim in sims:
            sim.llg_pass(V.PASS_CORRECTOR)
        refresh(V.STATE_SPIN)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("nranks", [2, 3])
def test_shards_equal_whole_system(vgpu_lib, prec, nranks):
    import torch
    from vampire_b200 import vgpu as V
    s = S.config_fcc_tensor(L=6, seed=3)           # 864 spins, tensor + DMI, 2 materials, T = 300 K
    plans = SH.make_plan(s, nranks)
    dtype = torch.float32 if prec == "fp32" else torch.float64
    sims, masks = [], []
    try:
        for p in plans:
            loc = SH.local_system(s, p)
            sim = V.Simulation(loc, precision=prec, noise_seed=9)
            sim.set_owned(p.n_owned, p.noise_base)
            masks.append(sim.add_mask(*loc.masks["material"]))
            sims.append(sim)
        steps = 12
        _step_shards(V, torch, plans, sims, steps, dtype)
        with V.Simulation(s, precision=prec, noise_seed=9) as whole:
            wid = whole.add_mask(*s.masks["material"])
            whole.llg_heun(steps)
            ref = whole.spins()
            whole.stats_update(magnetization=True)
            m_whole, _, _ = whole.magnetization(wid)
        got = np.zeros_like(ref)
        for sim, p in zip(sims, plans):
            got[:, p.owned] = sim.spins()[:, :p.n_owned]
        np.testing.assert_array_equal(got, ref)
        size = s.masks["material"][1]
        total = np.zeros((size, 8))
        for sim, mid in zip(sims, masks):
            sim.stats_update(magnetization=True)
            total += sim.stats_sums(mid, size)
        comb = SH.combine_magnetization(total[:, :4])
        np.testing.assert_allclose(comb.ravel(), np.asarray(m_whole).reshape(-1)[: comb.size], rtol=1e-10, atol=1e-12)
    finally:
        for sim in sims:
            sim.close()


def test_shard_setup_order_is_checked(vgpu_lib):
    """Monte Carlo colour lists follow the owned count given before
    vgpu_mc_setup: changing it afterwards is refused, as is an owned count
    beyond the local atoms."""
    from vampire_b200 import vgpu as V
    s = S.config_fcc_tensor(L=3, seed=3)
    p = SH.make_plan(s, 2)[0]
    with V.Simulation(SH.local_system(s, p)) as sim:
        sim.set_owned(p.n_owned, p.noise_base)
        sim.mc_setup()
        with pytest.raises(V.VGPUError) as e:
            sim.set_owned(p.n_owned - 1, p.noise_base)
        assert e.value.code == V.ERR_STATE
        with pytest.raises(V.VGPUError):
            sim.set_owned(p.n_local + 1, 0)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("nranks", [2, 3])
def test_mc_shards_equal_whole_system(vgpu_lib, prec, nranks):
    """Monte Carlo on shards (the whole system's colouring restricted to each
    shard, one vgpu_mc_colour per colour with a halo refresh between) equals
    the whole system's sweeps bit for bit: owned spins and the summed move
    and rejection counters."""
    import torch
    from vampire_b200 import vgpu as V
    s = S.config_fcc_tensor(L=6, seed=3, temperature=600.0)
    plans = SH.make_plan(s, nranks)
    dtype = torch.float32 if prec == "fp32" else torch.float64
    sweeps = 6
    with V.Simulation(s, precision=prec, noise_seed=21) as whole:
        nc = whole.mc_setup()
        colour = whole.mc_colours()
        whole.mc_sweep(sweeps)
        ref = whole.spins()
        moves_w, rej_w = whole.mc_counters()
    sims = []
    try:
        for p in plans:
            sim = V.Simulation(SH.local_system(s, p), precision=prec, noise_seed=21)
            sim.set_owned(p.n_owned, p.noise_base)
            assert sim.mc_setup(SH.local_colours(colour, p)) == nc
            sims.append(sim)
        refresh = _refresher(torch, plans, sims, dtype)
        for _ in range(sweeps):
            SH.mc_sweep_sharded(nc, lambda c: [sim.mc_colour(c) for sim in sims], lambda: refresh(V.STATE_SPIN))
        got = np.zeros_like(ref)
        moves = rej = 0.0
        for sim, p in zip(sims, plans):
            got[:, p.owned] = sim.spins()[:, :p.n_owned]
            mv, rj = sim.mc_counters()
            moves += mv
            rej += rj
        np.testing.assert_array_equal(got, ref)
        assert moves == moves_w == sweeps * s.n and rej == rej_w and 0 < rej < moves
        with pytest.raises(V.VGPUError) as e:
            sims[0].mc_colour(1)          # a sweep starts with colour 0
        assert e.value.code == V.ERR_ARG
    finally:
        for sim in sims:
            sim.close()


def _sum_moments(torch, sims):
    """Host stand-in for the all-reduce of the shards' cell moments: add the
    device buffers of every shard and write the sum back into each."""
    bufs = [sim.dipole_moment_tensor() for sim in sims]
    for sim in sims:
        sim.synchronize()
    total = torch.stack(bufs).sum(0)
    for b in bufs:
        b.copy_(total)
    torch.cuda.synchronize()
    for sim in sims:
        sim.dipole_finish()


@pytest.mark.parametrize("solver", ["tensor", "macrocell"])
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("nranks", [2, 3])
def test_dipole_shards_equal_whole_system(vgpu_lib, solver, prec, nranks):
    """The macrocell dipole field on shards: each shard sums its owned atoms
    into the cell moments, the host adds them over shards, and the cell fields
    and the trajectory across dipole updates equal the whole system's (up to
    the order of the moment additions).  A pass while the field awaits the sum
    is refused."""
    import torch
    from vampire_b200 import vgpu as V
    s = S.config_fcc_tensor(L=6, seed=3)
    cells = S.dipole_cells(s, size=2 * 3.54, atomic_volume=3.54 ** 3 / 4, solver=solver, update_rate=4)
    plans = SH.make_plan(s, nranks)
    dtype = torch.float32 if prec == "fp32" else torch.float64
    steps = 10
    with V.Simulation(s, precision=prec, noise_seed=5) as whole:
        whole.dipole_setup(cells)
        m0, b0, h0 = whole.dipole_cells()
        whole.llg_heun(steps)
        ref = whole.spins()
        m1, b1, _ = whole.dipole_cells()
    assert np.abs(b0).max() > 0
    sims = []
    try:
        for p in plans:
            sim = V.Simulation(SH.local_system(s, p), precision=prec, noise_seed=5)
            sim.set_owned(p.n_owned, p.noise_base)
            sim.dipole_setup_shard(cells, s.type, np.concatenate([p.owned, p.halo]))
            assert sim.dipole_pending()
            sims.append(sim)
        with pytest.raises(V.VGPUError) as e:
            sims[0].llg_pass(V.PASS_PREDICTOR)
        assert e.value.code == V.ERR_STATE
        _sum_moments(torch, sims)
        for sim in sims:
            assert not sim.dipole_pending()
            m, b, h = sim.dipole_cells()
            assert np.abs(m - m0).max() <= 1e-14 * np.abs(m0).max()
            assert np.abs(b - b0).max() <= 1e-6 * np.abs(b0).max()
            assert np.abs(h - h0).max() <= 1e-6 * np.abs(h0).max()
        refresh = _refresher(torch, plans, sims, dtype)
        for _ in range(steps):
            for sim in sims:
                sim.llg_pass(V.PASS_PREDICTOR)
            refresh(V.STATE_PREDICTOR)
            for sim in sims:
                sim.llg_pass(V.PASS_CORRECTOR)
            refresh(V.STATE_SPIN)
            if sims[0].dipole_pending():
                _sum_moments(torch, sims)
        got = np.zeros_like(ref)
        for sim, p in zip(sims, plans):
            got[:, p.owned] = sim.spins()[:, :p.n_owned]
            _, b, _ = sim.dipole_cells()
            assert np.abs(b - b1).max() <= 1e-5 * np.abs(b1).max()
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-5 if prec == "fp32" else 1e-11)
    finally:
        for sim in sims:
            sim.close()


def _step_shards_overlapped(V, torch, plans, sims, ranges, steps, dtype):
    """The overlapped order on one GPU: every shard's core range, the halo
    refresh (host-driven), then the boundary ranges, for each pass."""
    refresh = _refresher(torch, plans, sims, dtype)
    for _ in range(steps):
        for which, state in ((V.PASS_PREDICTOR, V.STATE_SPIN), (V.PASS_CORRECTOR, V.STATE_PREDICTOR)):
            for sim, rg in zip(sims, ranges):
                if rg is not None:
                    sim.llg_pass_range(which, *rg[0])
            refresh(state)
            for sim, rg, p in zip(sims, ranges, plans):
                for a, b in (rg[1] if rg is not None else [(0, p.n_owned)]):
                    sim.llg_pass_range(which, a, b)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("nranks", [2, 3])
def test_range_passes_equal_whole_system(vgpu_lib, prec, nranks):
    """vgpu_llg_pass_range: shards stepped core range first, boundary ranges
    after the halo refresh (the overlapped order), staged FP32 passes
    included, equal the whole system on one handle bit for bit; the step
    counter advances once per step."""
    import torch
    from vampire_b200 import vgpu as V
    s = S.config_fcc_tensor(L=12, seed=3)          # 6912 spins, tensor + DMI, 2 materials, T = 300 K
    plans = SH.make_plan(s, nranks)
    dtype = torch.float32 if prec == "fp32" else torch.float64
    sims, ranges = [], []
    try:
        for p in plans:
            loc = SH.local_system(s, p)
            sim = V.Simulation(loc, precision=prec, noise_seed=9)
            sim.set_owned(p.n_owned, p.noise_base)
            sims.append(sim)
            ranges.append(SH.split_ranges(loc, p.n_owned))
        assert all(r is not None for r in ranges)
        steps = 8
        _step_shards_overlapped(V, torch, plans, sims, ranges, steps, dtype)
        assert all(sim.step == steps for sim in sims)
        with V.Simulation(s, precision=prec, noise_seed=9) as whole:
            whole.llg_heun(steps)
            ref = whole.spins()
        got = np.zeros_like(ref)
        for sim, p in zip(sims, plans):
            got[:, p.owned] = sim.spins()[:, :p.n_owned]
        np.testing.assert_array_equal(got, ref)
    finally:
        for sim in sims:
            sim.close()


def test_range_pass_arguments_checked(vgpu_lib):
    from vampire_b200 import vgpu as V
    s = S.config_fcc_tensor(L=3, seed=3)
    with V.Simulation(s) as sim:
        for first, end in ((16, 64), (0, s.n + 1), (64, 32), (-32, 0)):
            with pytest.raises(V.VGPUError) as e:
                sim.llg_pass_range(V.PASS_PREDICTOR, first, end)
            assert e.value.code == V.ERR_ARG


def _one_rank_main(rank, port, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        from vampire_b200 import vgpu as V
        s = S.config_fcc_tensor(L=6, seed=3)
        plan = SH.make_plan(s, 1)[0]
        sh = SH.ShardedSimulation(s, plan, device=0, noise_seed=9)
        assert sh.ranges is not None
        sh.step(6)
        got = sh.owned_spins()
        with V.Simulation(s, noise_seed=9) as whole:
            whole.llg_heun(6)
            ref = whole.spins()
        np.save(out, np.abs(got - ref).max())
        sh.sim.close()
    finally:
        dist.destroy_process_group()


def test_sharded_simulation_one_rank_nccl(vgpu_lib, tmp_path):
    """ShardedSimulation over a one-rank NCCL group: the overlapped step
    (communication stream, events, core and boundary ranges) with no peers
    equals the whole system bit for bit."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    out = str(tmp_path / "dev.npy")
    mp.start_processes(_one_rank_main, args=(port, out), nprocs=1, join=True, start_method="spawn")
    assert float(np.load(out)) == 0.0
