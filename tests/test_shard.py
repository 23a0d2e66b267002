"""Spatial sharding host logic (vampire_b200/shard.py) on CPU.

The plan and local systems are checked structurally; the halo exchange runs
as world_size-2, -3 and -4 gloo process groups whose ranks step their shard with
the FP64 oracle (predictor half, halo refresh of s', corrector half, halo
refresh of s) and must reproduce the whole-system oracle bit for bit -- the
same field sums in the same bond order, with the reference's replayed noise.
Monte Carlo shards run each colour's Metropolis pass over their owned atoms
with a halo refresh after every colour, against the whole-system sweep.
"""
import os
import socket

import numpy as np
import pytest

from vampire_b200 import shard as SH
from vampire_b200 import system as S


def _fcc(L=4, T=300.0):
    return S.config_fcc_tensor(L=L, seed=11, temperature=T)


def _sc_open():
    mats = [S.Material(alpha=0.1, mu_s_muB=1.72, Ku=6.69e-24)]
    p = S.SimParams(dt_SI=1e-16, temperature=0.0, H_applied=0.1, H_vec=(0.0, 0.0, 1.0))
    return S.build("sc", 5, 4, 7, 3.0, mats, np.array([[11.2e-21]]), p, periodic=(False, True, False), spin_seed=3)


@pytest.mark.parametrize("by", ["index", "z", "x"])
@pytest.mark.parametrize("nranks", [1, 2, 3, 4])
@pytest.mark.parametrize("maker", [_fcc, _sc_open])
def test_plan_covers_system_and_halos_are_consistent(maker, nranks, by):
    s = maker()
    plans = SH.make_plan(s, nranks, by=by)
    owned = np.concatenate([p.owned for p in plans])
    assert np.array_equal(np.sort(owned), np.arange(s.n))          # a partition
    owner = np.empty(s.n, dtype=int)
    for p in plans:
        owner[p.owned] = p.rank
    for p in plans:
        # halo = exactly the non-owned neighbours of owned atoms
        need = set()
        for i in p.owned:
            for j in s.nl[s.nl_start[i]:s.nl_end[i] + 1]:
                if owner[j] != p.rank:
                    need.add(int(j))
        assert set(p.halo.tolist()) == need
        # every halo block matches what its source rank sends, in order
        for src, (first, count) in p.recv.items():
            sent = plans[src].send[p.rank]
            assert sent.size == count
            assert np.array_equal(plans[src].owned[sent], p.halo[first - p.n_owned:first - p.n_owned + count])
        loc = SH.local_system(s, p)
        assert loc.n == p.n_local
        assert np.all(loc.nl_end[p.n_owned:] < loc.nl_start[p.n_owned:])  # halo rows empty
        glob = np.concatenate([p.owned, p.halo])
        for k in range(0, p.n_owned, max(1, p.n_owned // 17)):
            g = p.owned[k]
            mine = glob[loc.nl[loc.nl_start[k]:loc.nl_end[k] + 1]]
            assert np.array_equal(mine, s.nl[s.nl_start[g]:s.nl_end[g] + 1])


@pytest.mark.parametrize("nranks", [2, 3, 5])
def test_index_shares_give_noise_base(nranks):
    s = _fcc(L=3)
    for p in SH.make_plan(s, nranks):
        assert p.noise_base == int(p.owned[0])


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _rank_main(rank, world, port, maker_name, steps, seed, out_dir):
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        s = {"fcc": _fcc, "sc": _sc_open}[maker_name]()
        plan = SH.make_plan(s, world)[rank]
        loc = SH.local_system(s, plan)
        o = O.OracleSystem(loc)
        glob = np.concatenate([plan.owned, plan.halo])
        rng = np.random.default_rng(seed)
        xi_all = rng.standard_normal((steps, 3, s.n))
        ex = SH.HaloExchange(plan)
        state = {"cur": None}

        def pack(peer, idx):
            return torch.from_numpy(np.ascontiguousarray(state["cur"][:, idx]).ravel())

        def unpack(peer, first, count, buf):
            state["cur"][:, first:first + count] = buf.numpy().reshape(3, count)

        def alloc(k):
            return torch.empty(k, dtype=torch.float64)

        spins = loc.spins.copy()
        for t in range(steps):
            xi = xi_all[t][:, glob].ravel()
            p, keep = o.heun_predict(spins, xi)
            state["cur"] = p
            ex.exchange(pack, unpack, alloc)
            spins = o.heun_correct(spins, p, keep)
            state["cur"] = spins
            ex.exchange(pack, unpack, alloc)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), spins[:, :plan.n_owned])
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _rank_main_overlap(rank, world, port, maker_name, steps, seed, out_dir):
    """As _rank_main, in the overlapped order of ShardedSimulation.step: each
    pass posts the exchange of its input state, updates the core atoms while
    the halo still holds the previous values, completes the exchange, then
    updates the boundary ranges.  A pass over a range is the oracle's pass of
    the whole shard with only that range's atoms taken."""
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        s = {"fcc": _fcc, "sc": _sc_open, "fcc_big": lambda: _fcc(L=12)}[maker_name]()
        plan = SH.make_plan(s, world)[rank]
        loc = SH.local_system(s, plan)
        o = O.OracleSystem(loc)
        n = loc.n
        glob = np.concatenate([plan.owned, plan.halo])
        rng = np.random.default_rng(seed)
        xi_all = rng.standard_normal((steps, 3, s.n))
        ex = SH.HaloExchange(plan)
        ranges = SH.split_ranges(loc, plan.n_owned)
        assert ranges is not None or maker_name != "fcc_big"
        # no core range: nothing runs during the exchange
        order = [ranges[0]] + ranges[1] if ranges else [(0, 0), (0, plan.n_owned)]
        state = {"s": loc.spins.copy(), "p": loc.spins.copy()}

        def exchange(key, run):
            cur = state[key]
            pend = ex.begin(lambda peer, idx: torch.from_numpy(np.ascontiguousarray(cur[:, idx]).ravel()),
                            lambda k: torch.empty(k, dtype=torch.float64))
            run(order[0])                   # core: the halo still holds the old values
            def unpack(peer, first, count, buf):
                cur[:, first:first + count] = buf.numpy().reshape(3, count)
            ex.end(pend, unpack)
            for r in order[1:]:
                run(r)

        keep = np.zeros((12, n))
        for t in range(steps):
            xi = xi_all[t][:, glob].ravel()

            def predict(r):
                p, k = o.heun_predict(state["s"], xi)
                state["p"][:, r[0]:r[1]] = p[:, r[0]:r[1]]
                keep[:, r[0]:r[1]] = k.reshape(12, n)[:, r[0]:r[1]]

            def correct(r):
                s1 = o.heun_correct(state["s"], state["p"], keep.ravel().copy())
                state["s"][:, r[0]:r[1]] = s1[:, r[0]:r[1]]

            exchange("s", predict)
            exchange("p", correct)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), state["s"][:, :plan.n_owned])
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_split_ranges_core_needs_no_halo():
    """The core range's atoms read no halo atom; the ranges tile the owned
    atoms; core and boundary cuts fall on slice (32-atom) boundaries; the last
    range ends at the owned count."""
    s = _fcc(L=12)
    for world in (2, 3, 4):
        for plan in SH.make_plan(s, world):
            loc = SH.local_system(s, plan)
            (c0, c1), bnd = SH.split_ranges(loc, plan.n_owned)
            assert c0 % 32 == 0 and c1 % 32 == 0 and c1 > c0
            for i in range(c0, c1):
                assert np.all(loc.nl[loc.nl_start[i]:loc.nl_end[i] + 1] < plan.n_owned)
            cover = sorted([(c0, c1)] + bnd)
            assert cover[0][0] == 0 and cover[-1][1] == plan.n_owned
            assert all(a[1] == b[0] for a, b in zip(cover, cover[1:]))
            assert bnd[-1][1] == plan.n_owned


@pytest.mark.parametrize("maker_name,world", [("fcc_big", 2), ("fcc_big", 3), ("fcc_big", 4)])
def test_gloo_overlapped_shards_equal_whole_system(tmp_path, maker_name, world):
    """The overlapped schedule (core range during the exchange) reproduces
    the whole-system oracle bit for bit over 4 stochastic steps."""
    import torch.multiprocessing as mp
    from oracle import oracle as O
    steps, seed = 4, 5
    mp.start_processes(_rank_main_overlap, args=(world, _free_port(), maker_name, steps, seed, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    s = _fcc(L=12)
    rng = np.random.default_rng(seed)
    xi_all = rng.standard_normal((steps, 3, s.n))
    o = O.OracleSystem(s)
    ref = s.spins.copy()
    for t in range(steps):
        ref = o.llg_heun(ref, 1, xi=xi_all[t].ravel())
    got = np.zeros_like(ref)
    for plan in SH.make_plan(s, world):
        got[:, plan.owned] = np.load(tmp_path / f"rank{plan.rank}.npy")
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("maker_name,world", [("fcc", 2), ("sc", 3)])
def test_gloo_sharded_oracle_equals_whole_system(tmp_path, maker_name, world):
    import torch.multiprocessing as mp
    from oracle import oracle as O
    steps, seed = 5, 7
    mp.start_processes(_rank_main, args=(world, _free_port(), maker_name, steps, seed, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    s = {"fcc": _fcc, "sc": _sc_open}[maker_name]()
    rng = np.random.default_rng(seed)
    xi_all = rng.standard_normal((steps, 3, s.n))
    whole = O.OracleSystem(s).llg_heun(s.spins, steps, xi_all.reshape(steps, -1).ravel())
    plans = SH.make_plan(s, world)
    got = np.zeros_like(whole)
    for p in plans:
        got[:, p.owned] = np.load(tmp_path / f"rank{p.rank}.npy")
    np.testing.assert_array_equal(got, whole)


def _greedy_colours(s):
    colour = np.full(s.n, -1)
    for i in range(s.n):
        used = {colour[j] for j in s.nl[s.nl_start[i]:s.nl_end[i] + 1]}
        c = 0
        while c in used:
            c += 1
        colour[i] = c
    return colour


def _mc_rank_main(rank, world, port, maker_name, sweeps, seed, out_dir):
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        s = _fcc(T=600.0) if maker_name == "fcc" else _sc_open()
        colour = _greedy_colours(s)
        plan = SH.make_plan(s, world)[rank]
        loc = SH.local_system(s, plan)
        o = O.OracleSystem(loc)
        glob = np.concatenate([plan.owned, plan.halo])
        lcol = SH.local_colours(colour, plan)
        rnd_all = _mc_numbers(s.n, sweeps, seed)
        ex = SH.HaloExchange(plan)
        state = {"cur": loc.spins.copy()}

        def pack(peer, idx):
            return torch.from_numpy(np.ascontiguousarray(state["cur"][:, idx]).ravel())

        def unpack(peer, first, count, buf):
            state["cur"][:, first:first + count] = buf.numpy().reshape(3, count)

        def alloc(k):
            return torch.empty(k, dtype=torch.float64)

        rejects = 0
        for t in range(sweeps):
            rnd = rnd_all[t][:, glob].ravel()

            def run_colour(c):
                nonlocal rejects
                atoms = np.flatnonzero(lcol[:plan.n_owned] == c)
                state["cur"], r = o.mc_pass(state["cur"], atoms, rnd)
                rejects += r

            SH.mc_sweep_sharded(int(colour.max()) + 1, run_colour, lambda: ex.exchange(pack, unpack, alloc))
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), state["cur"][:, :plan.n_owned])
        np.save(os.path.join(out_dir, f"rej{rank}.npy"), np.array([rejects]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _mc_numbers(n, sweeps, seed):
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((sweeps, 3, n))
    u = rng.random((sweeps, 1, n))
    return np.concatenate([g, u], axis=1)


@pytest.mark.parametrize("maker_name,world", [("fcc", 2), ("sc", 3), ("fcc", 4)])
def test_gloo_sharded_monte_carlo_equals_whole_system(tmp_path, maker_name, world):
    """Colour-ordered Metropolis sweeps on shards (owned atoms of one colour,
    then a halo refresh, for every colour) reproduce the whole system's
    sweeps bit for bit with the FP64 oracle and the same random numbers, and
    the shards' rejections add up to the whole system's."""
    import torch.multiprocessing as mp
    from oracle import oracle as O
    sweeps, seed = 4, 5
    mp.start_processes(_mc_rank_main, args=(world, _free_port(), maker_name, sweeps, seed, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    s = _fcc(T=600.0) if maker_name == "fcc" else _sc_open()
    colour = _greedy_colours(s)
    o = O.OracleSystem(s)
    spins, rejects = s.spins.copy(), 0
    for t, rnd in enumerate(_mc_numbers(s.n, sweeps, seed)):
        spins, r = o.mc_colour_sweep(spins, colour, rnd.ravel())
        rejects += r
    got = np.zeros_like(spins)
    rej = 0
    for p in SH.make_plan(s, world):
        got[:, p.owned] = np.load(tmp_path / f"rank{p.rank}.npy")
        rej += int(np.load(tmp_path / f"rej{p.rank}.npy")[0])
    np.testing.assert_array_equal(got, spins)
    assert rej == rejects and 0 < rejects < sweeps * s.n


def test_combined_magnetization_equals_whole_system():
    s = _fcc(L=4)
    mask, size = s.masks["material"]
    mu = s.mu_s_muB()
    whole = np.zeros((size, 4))
    for q in range(3):
        np.add.at(whole[:, q], mask, mu * s.spins[q])
    np.add.at(whole[:, 3], mask, mu)
    parts = np.zeros((size, 4))
    for p in SH.make_plan(s, 3):
        loc = SH.local_system(s, p)
        lm, _ = loc.masks["material"]
        lmu = loc.mu_s_muB()
        o = slice(0, p.n_owned)
        for q in range(3):
            np.add.at(parts[:, q], lm[o], lmu[o] * loc.spins[q][o])
        np.add.at(parts[:, 3], lm[o], lmu[o])
    np.testing.assert_allclose(SH.combine_magnetization(parts), SH.combine_magnetization(whole), rtol=1e-13)


def _dipole_rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    from oracle import dipole_ref as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        s = _fcc()
        cells = S.dipole_cells(s, size=2 * 3.54, atomic_volume=3.54 ** 3 / 4, solver="tensor", update_rate=1)
        plan = SH.make_plan(s, world)[rank]
        nc = cells["cell_natoms"].size
        own = plan.owned
        part = D.cell_moments(s.spins[:, own], s.materials["mu_s_SI"][s.type[own]], cells["atom_cell"][own], nc)
        buf = torch.from_numpy(np.ascontiguousarray(part).ravel())
        SH.sum_cell_moments(buf)
        np.save(os.path.join(out_dir, f"mag{rank}.npy"), buf.numpy().reshape(3, nc))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 4])
def test_gloo_sharded_cell_moments_equal_whole_system(tmp_path, world):
    """Macrocell moments on shards: every rank sums its owned atoms, one
    all-reduce adds the partial moments (cells::mag's MPI_Allreduce), and
    every rank holds the whole system's moments -- equal to the whole-system
    sum up to the order of the additions -- and so the same cell fields."""
    import torch.multiprocessing as mp
    from oracle import dipole_ref as D
    mp.start_processes(_dipole_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    s = _fcc()
    c = S.dipole_cells(s, size=2 * 3.54, atomic_volume=3.54 ** 3 / 4, solver="tensor", update_rate=1)
    nc = c["cell_natoms"].size
    whole = D.cell_moments(s.spins, s.materials["mu_s_SI"][s.type], c["atom_cell"], nc)
    T = D.tensors(c["cell_pos_mom"], c["cell_natoms"], c["macro_cell_size"], c["cutoff"], "tensor", s.coords,
                  c["atom_cell"])
    B0, H0 = D.cell_fields(whole, T, c["cell_natoms"], c["cell_volume"])
    scale = np.abs(whole).max()
    assert scale > 0
    for r in range(world):
        mag = np.load(tmp_path / f"mag{r}.npy")
        assert np.abs(mag - whole).max() <= 1e-14 * scale
        B, H = D.cell_fields(mag, T, c["cell_natoms"], c["cell_volume"])
        assert np.abs(B - B0).max() <= 1e-13 * np.abs(B0).max()
        assert np.abs(H - H0).max() <= 1e-13 * np.abs(H0).max()


def test_cell_moment_sum_without_process_group_is_the_single_shard():
    """One shard and no process group (a single-GPU run of the sharded
    path): the partial cell moments are already the whole system's."""
    import torch
    import torch.distributed as dist
    from vampire_b200 import shard as SH
    assert not dist.is_initialized()
    buf = torch.arange(6, dtype=torch.float64)
    SH.sum_cell_moments(buf)
    assert torch.equal(buf, torch.arange(6, dtype=torch.float64))
