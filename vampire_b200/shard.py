"""Spatial sharding of one spin system over ranks (one process per GPU).

The reference distributes a system over MPI ranks by space: each rank owns
the atoms of its sub-domain ("core" and "boundary" atoms) and keeps copies of
the neighbouring ranks' boundary atoms ("halo"), refreshed before every field
evaluation (src/simulate/LLGHeun-mpi.cpp:62-64, src/mpi/mpi_comms.cpp:45-143).
The same decomposition here, one process per GPU over NVLink/NCCL:

* ``make_plan`` cuts the system into ``nranks`` shares of equal atom count
  (contiguous atom-index ranges, or slabs along one axis) and, for every rank, lists its
  owned atoms, its halo atoms grouped by owning rank, and for every peer the
  owned atoms that peer holds as halo (in the peer's halo order).  Every rank
  computes the same plan from the same system, so no plan is exchanged.
* ``local_system`` renumbers a rank's share: owned atoms first (global
  order), then halo atoms by source rank.  Owned atoms keep their bonds
  (neighbour indices renumbered, bond order and couplings unchanged, so the
  field of an owned atom is the same sum in the same order as in the whole
  system); halo atoms carry no bonds -- their spins are inputs only.
* ``HaloExchange`` moves the boundary spins between the two passes of a Heun
  step: one send and one receive per peer (three components packed into one
  message), posted together with ``torch.distributed.batch_isend_irecv``.
  It works with CPU tensors over gloo (tests) and device tensors over NCCL.
* ``ShardedSimulation`` drives one rank's shard on its GPU.  Every pass
  starts the halo exchange of its input state (s for the predictor, s' for
  the corrector) on a communication stream, runs the shard's core atoms --
  the owned atoms whose neighbours are all owned (``split_ranges``) -- on the
  library's stream meanwhile, then, once the exchange has landed, the
  boundary atoms: the reference's mpi_init_halo_swap / core update /
  mpi_complete_halo_swap / boundary update (src/mpi/LLGHeun-mpi.cpp:61-140).
  The fused passes update the owned atoms only (``vgpu_set_owned``) and key
  the thermal noise by global atom index, so a sharded run draws the same
  noise as one GPU.

Statistics combine across ranks from the raw per-bin sums of each shard
(``vgpu_stats_get_sums``) with one all-reduce.

The macrocell dipole field shards as the reference's does: every rank sums
its owned atoms into the cell moments, one all-reduce adds them over ranks
(cells::mag's MPI_Allreduce, src/cells/mag.cpp:69-74), and every rank then
computes the cell fields from the sums (``sum_cell_moments``,
``ShardedSimulation.dipole_setup``).

Monte Carlo shards the same way.  A colour-ordered Metropolis sweep updates
one colour at a time; a shard runs its owned atoms of a colour, then every
rank refreshes its halo spins before the next colour (``mc_sweep_sharded``),
as the reference's parallel Monte Carlo swaps halos around each of its eight
octant phases (src/montecarlo/mc-mpi.cpp:140-210).  With the whole system's
colouring and the move random numbers keyed by global atom index, the shards
together make exactly the whole system's sweep.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

from .system import SpinSystem


@dataclass
class ShardPlan:
    rank: int
    nranks: int
    owned: np.ndarray                     # global ids of owned atoms (ascending)
    halo: np.ndarray                      # global ids of halo atoms, grouped by source rank
    recv: Dict[int, Tuple[int, int]]      # peer -> (first local index, count) of its halo block
    send: Dict[int, np.ndarray]           # peer -> local indices of owned atoms it holds as halo
    noise_base: Optional[int]             # global id of owned[0] when owned is one contiguous range

    @property
    def n_owned(self) -> int:
        return int(self.owned.size)

    @property
    def n_local(self) -> int:
        return int(self.owned.size + self.halo.size)


def _owner_slabs(s: SpinSystem, nranks: int, by: str) -> np.ndarray:
    """Owner rank of every atom.  by="index": equal contiguous ranges of atom
    index (cell layers for lattices numbered cell by cell along z, as the
    builders and the reference's unit-cell loops do; a shard's noise then
    follows the whole system's Philox stream); by="x"|"y"|"z": equal-count
    slabs along that coordinate (ties broken by atom index)."""
    n = s.n
    if by == "index" or s.coords is None:
        order = np.arange(n)
    else:
        order = np.lexsort((np.arange(n), s.coords["xyz".index(by)]))
    owner = np.empty(n, dtype=np.int32)
    bounds = np.linspace(0, n, nranks + 1).round().astype(np.int64)
    for r in range(nranks):
        owner[order[bounds[r]:bounds[r + 1]]] = r
    return owner


def make_plan(s: SpinSystem, nranks: int, by: str = "index") -> List[ShardPlan]:
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    if by not in ("index", "x", "y", "z"):
        raise ValueError("by must be 'index', 'x', 'y' or 'z'")
    n = s.n
    owner = _owner_slabs(s, nranks, by)
    deg = (s.nl_end - s.nl_start + 1).astype(np.int64)
    src = np.repeat(np.arange(n), deg)                    # bond -> atom
    nbr = s.nl.astype(np.int64)
    # (rank r needs atom j as halo) for bonds i -> j with owner[i] = r != owner[j]
    cross = owner[src] != owner[nbr]
    need = {r: set() for r in range(nranks)}
    for r, j in zip(owner[src[cross]], nbr[cross]):
        need[int(r)].add(int(j))
    plans = []
    owned_of = [np.flatnonzero(owner == r) for r in range(nranks)]
    halo_of = {}
    for r in range(nranks):
        h = np.array(sorted(need[r], key=lambda j: (owner[j], j)), dtype=np.int64)
        halo_of[r] = h
    for r in range(nranks):
        own = owned_of[r]
        h = halo_of[r]
        recv = {}
        first = own.size
        for p in range(nranks):
            cnt = int(np.count_nonzero(owner[h] == p)) if h.size else 0
            if cnt:
                recv[p] = (first, cnt)
                first += cnt
        send = {}
        pos = {int(g): k for k, g in enumerate(own)}
        for p in range(nranks):
            if p == r:
                continue
            hp = halo_of[p]
            mine = hp[owner[hp] == r] if hp.size else hp
            if mine.size:
                send[p] = np.array([pos[int(g)] for g in mine], dtype=np.int32)
        contiguous = own.size > 0 and int(own[-1]) - int(own[0]) + 1 == own.size
        plans.append(ShardPlan(rank=r, nranks=nranks, owned=own, halo=h, recv=recv, send=send,
                               noise_base=int(own[0]) if contiguous else None))
    return plans


def local_system(s: SpinSystem, plan: ShardPlan) -> SpinSystem:
    """The rank's share of `s`: owned atoms (with their bonds) then halo atoms
    (no bonds), neighbour indices renumbered locally."""
    glob = np.concatenate([plan.owned, plan.halo]).astype(np.int64)
    loc = np.full(s.n, -1, dtype=np.int64)
    loc[glob] = np.arange(glob.size)
    n_own, n_loc = plan.n_owned, plan.n_local
    st = s.nl_start[plan.owned].astype(np.int64)
    en = s.nl_end[plan.owned].astype(np.int64)
    deg = en - st + 1
    bonds = np.concatenate([np.arange(a, b + 1) for a, b in zip(st, en)]) if n_own else np.zeros(0, np.int64)
    nl = loc[s.nl[bonds]]
    if (nl < 0).any():
        raise AssertionError("halo plan misses a neighbour")
    start = np.zeros(n_loc, dtype=np.int32)
    end = np.zeros(n_loc, dtype=np.int32)
    off = np.concatenate([[0], np.cumsum(deg)])
    start[:n_own] = off[:-1]
    end[:n_own] = off[1:] - 1
    start[n_own:] = off[-1]           # halo atoms: empty rows (end = start - 1)
    end[n_own:] = off[-1] - 1
    if s.nl_type is not None:
        nl_type = s.nl_type[bonds].astype(np.int32)
        jlist = s.jlist
    else:
        w = {0: 1, 1: 3, 2: 9}[s.exch_type]
        nl_type = None
        jlist = s.jlist.reshape(-1, w)[bonds].ravel() if w > 1 else s.jlist[bonds]
    masks = {k: (np.asarray(m)[glob].astype(np.int32), size) for k, (m, size) in s.masks.items()}
    aniso = None
    if s.aniso is not None:
        aniso = dict(s.aniso)
        if aniso.get("neel_tensor") is not None:
            aniso["neel_tensor"] = np.ascontiguousarray(aniso["neel_tensor"][glob])
    return SpinSystem(n=n_loc, nl_start=start, nl_end=end, nl=nl.astype(np.int32), jlist=jlist,
                      exch_type=s.exch_type, type=s.type[glob].astype(np.int32), materials=s.materials,
                      spins=np.ascontiguousarray(s.spins[:, glob]), params=s.params, uniaxial=s.uniaxial,
                      cubic=s.cubic, nl_type=nl_type,
                      coords=None if s.coords is None else np.ascontiguousarray(s.coords[:, glob]),
                      masks=masks, cells=None, aniso=aniso)


def split_ranges(loc: SpinSystem, n_owned: int):
    """Atom ranges of a shard's overlapped passes: (core, boundary) with core =
    (c0, c1) the longest run of owned atoms whose neighbours are all owned
    (atoms n_owned.. are the halo), cut to multiples of 32 (slice boundaries),
    and boundary = the ranges before and after it, the last one ending at
    n_owned (the corrector range that completes the step runs last).  None
    when no core range of at least one slice exists."""
    if n_owned <= 0:
        return None
    deg = (loc.nl_end[:n_owned] - loc.nl_start[:n_owned] + 1).astype(np.int64)
    src = np.repeat(np.arange(n_owned), np.maximum(deg, 0))
    bonds = np.concatenate([np.arange(a, b + 1) for a, b in zip(loc.nl_start[:n_owned], loc.nl_end[:n_owned])
                            if b >= a]) if deg.sum() else np.zeros(0, np.int64)
    needs = np.zeros(n_owned, dtype=bool)
    if bonds.size:
        np.logical_or.at(needs, src, loc.nl[bonds] >= n_owned)
    best, start = (0, 0), None
    for i in range(n_owned + 1):
        if i < n_owned and not needs[i]:
            if start is None:
                start = i
        elif start is not None:
            if i - start > best[1] - best[0]:
                best = (start, i)
            start = None
    c0 = -(-best[0] // 32) * 32
    c1 = min(best[1] // 32 * 32, (n_owned - 1) // 32 * 32)
    if c1 <= c0:
        return None
    boundary = [(a, b) for a, b in ((0, c0), (c1, n_owned)) if b > a]
    return (c0, c1), boundary


class HaloExchange:
    """One halo refresh: for every peer, pack(peer, local_idx) -> tensor of
    3*count values is sent, and unpack(peer, first, count, tensor) receives
    the peer's block.  All sends and receives of a refresh are posted at once
    (torch.distributed.batch_isend_irecv), then waited for."""

    def __init__(self, plan: ShardPlan, group=None):
        self.plan = plan
        self.group = group

    def exchange(self, pack: Callable, unpack: Callable, alloc: Callable) -> None:
        import torch.distributed as dist
        ops, recv = [], {}
        for peer, (first, count) in sorted(self.plan.recv.items()):
            buf = alloc(3 * count)
            recv[peer] = (first, count, buf)
            ops.append(dist.P2POp(dist.irecv, buf, peer, self.group))
        for peer, idx in sorted(self.plan.send.items()):
            ops.append(dist.P2POp(dist.isend, pack(peer, idx), peer, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for peer, (first, count, buf) in recv.items():
            unpack(peer, first, count, buf)

    def begin(self, pack: Callable, alloc: Callable):
        """Post one refresh (every receive, then every send) and return its
        pending state; ``end`` completes it.  Work between the two must not
        read the halo atoms."""
        import torch.distributed as dist
        ops, recv, keep = [], {}, []
        for peer, (first, count) in sorted(self.plan.recv.items()):
            buf = alloc(3 * count)
            recv[peer] = (first, count, buf)
            ops.append(dist.P2POp(dist.irecv, buf, peer, self.group))
        for peer, idx in sorted(self.plan.send.items()):
            out = pack(peer, idx)
            keep.append(out)  # alive until the send completes
            ops.append(dist.P2POp(dist.isend, out, peer, self.group))
        reqs = dist.batch_isend_irecv(ops) if ops else []
        return reqs, recv, keep

    def end(self, pending, unpack: Callable) -> None:
        reqs, recv, _ = pending
        for req in reqs:
            req.wait()
        for peer, (first, count, buf) in recv.items():
            unpack(peer, first, count, buf)


def mc_sweep_sharded(ncolours: int, run_colour: Callable[[int], None], refresh: Callable[[], None]) -> None:
    """One Monte Carlo sweep of a shard: for every colour in order, the
    Metropolis pass over the shard's owned atoms of that colour, then the halo
    refresh of the spins (the next colour's sites read the moved neighbours).
    Every rank makes the same calls in the same order."""
    for c in range(ncolours):
        run_colour(c)
        refresh()


def local_colours(colour: np.ndarray, plan: ShardPlan) -> np.ndarray:
    """The whole system's colouring restricted to a shard's local atoms
    (owned, then halo), for vgpu_mc_setup on that shard."""
    return np.ascontiguousarray(np.asarray(colour)[np.concatenate([plan.owned, plan.halo])], dtype=np.int32)


def sum_cell_moments(buf, group=None) -> None:
    """Adds a shard's partial cell moments (a tensor of 3*ncells FP64, the
    owned atoms' sums) over all ranks in place: CPU tensors over gloo, the
    library's device buffer over NCCL.  Without a process group there is one
    shard, whose sums are already the whole system's."""
    import torch.distributed as dist
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)


def combine_magnetization(sums: np.ndarray) -> np.ndarray:
    """Reference normalisation (src/statistics/magnetization.cpp:134-180) of
    raw per-bin sums [bins, >=4] = (sum mu sx, sum mu sy, sum mu sz, sum mu)
    added over ranks: rows (m_hat_x, m_hat_y, m_hat_z, |m|/m_sat)."""
    out = np.zeros((sums.shape[0], 4))
    for b, v in enumerate(sums):
        msat = v[3]
        mag = np.sqrt(v[0] ** 2 + v[1] ** 2 + v[2] ** 2)
        if msat != 0.0:
            out[b] = (v[0] / mag, v[1] / mag, v[2] / mag, mag / msat)
    return out


class ShardedSimulation:
    """One rank's shard on its GPU (vampire_b200.vgpu over the C ABI), with
    NCCL halo exchange between the passes.  Collectives are issued on the
    library's stream, so the exchange is ordered after the pass that produced
    the boundary spins and before the pass that reads them."""

    def __init__(self, s: SpinSystem, plan: ShardPlan, device: int, precision: str = "fp32",
                 noise_seed: int = 0, group=None):
        import torch
        from . import vgpu
        self.plan = plan
        self.local = local_system(s, plan)
        self.sim = vgpu.Simulation(self.local, device=device, precision=precision, noise_seed=noise_seed)
        # non-contiguous shares draw their own (statistically equivalent) noise
        self.sim.set_owned(plan.n_owned, plan.noise_base if plan.noise_base is not None else 0)
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        self.device = torch.device("cuda", device)
        self.stream = torch.cuda.ExternalStream(self.sim.stream_ptr(), device=self.device)
        self.idx = {p: torch.as_tensor(ix, dtype=torch.int32, device=self.device) for p, ix in plan.send.items()}
        self.halo = HaloExchange(plan, group)
        # core atoms run while the exchange is in flight (on its own stream)
        self.ranges = split_ranges(self.local, plan.n_owned)
        self.comm = torch.cuda.Stream(device=self.device)
        self.group = group
        self._torch = torch
        self._global_type = np.ascontiguousarray(s.type, dtype=np.int32)
        self._moments = None

    def _refresh(self, which: int) -> None:
        torch = self._torch

        def pack(peer, _idx):
            ix = self.idx[peer]
            out = torch.empty(3 * ix.numel(), dtype=self.dtype, device=self.device)
            self.sim.halo_pack(which, ix.data_ptr(), ix.numel(), out.data_ptr())
            return out

        def unpack(peer, first, count, buf):
            self.sim.halo_unpack(which, first, count, buf.data_ptr())

        def alloc(k):
            return torch.empty(k, dtype=self.dtype, device=self.device)

        with torch.cuda.stream(self.stream):
            self.halo.exchange(pack, unpack, alloc)

    def dipole_setup(self, cells: dict) -> None:
        """The device dipole solver on this shard from the whole system's
        macrocells (system.dipole_cells of the whole system); every rank calls
        it, and the fields come from the moments summed over ranks."""
        self.sim.dipole_setup_shard(cells, self._global_type, np.concatenate([self.plan.owned, self.plan.halo]))
        self._moments = self.sim.dipole_moment_tensor()
        self._dipole_sum()

    def _dipole_sum(self) -> None:
        # every rank reaches the dipole cadence at the same step
        if self._moments is None or not self.sim.dipole_pending():
            return
        with self._torch.cuda.stream(self.stream):
            sum_cell_moments(self._moments, self.group)
        self.sim.dipole_finish()

    def _exchange_begin(self, which: int):
        """Start the halo exchange of state `which` on the communication
        stream, after everything on the library's stream so far."""
        torch = self._torch
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self.comm.wait_event(ev)
        comm = self.comm.cuda_stream

        def pack(peer, _idx):
            ix = self.idx[peer]
            out = torch.empty(3 * ix.numel(), dtype=self.dtype, device=self.device)
            self.sim.halo_pack_on(which, ix.data_ptr(), ix.numel(), out.data_ptr(), comm)
            return out

        def alloc(k):
            return torch.empty(k, dtype=self.dtype, device=self.device)

        with torch.cuda.stream(self.comm):
            return self.halo.begin(pack, alloc)

    def _exchange_end(self, which: int, pending) -> None:
        """Complete the exchange; the library's stream then waits for it."""
        torch = self._torch
        comm = self.comm.cuda_stream

        def unpack(peer, first, count, buf):
            self.sim.halo_unpack_on(which, first, count, buf.data_ptr(), comm)

        with torch.cuda.stream(self.comm):
            self.halo.end(pending, unpack)
            done = torch.cuda.Event()
            done.record(self.comm)
        self.stream.wait_event(done)

    def _pass(self, which_pass: int, input_state: int) -> None:
        if self.ranges is None:
            self._refresh(input_state)
            self.sim.llg_pass(which_pass)
            return
        (c0, c1), boundary = self.ranges
        pending = self._exchange_begin(input_state)
        self.sim.llg_pass_range(which_pass, c0, c1)
        self._exchange_end(input_state, pending)
        for a, b in boundary:
            self.sim.llg_pass_range(which_pass, a, b)

    def step(self, n_steps: int = 1) -> None:
        """Heun steps: each pass exchanges its input state's halo while the
        core atoms run, then runs the boundary atoms."""
        from . import vgpu
        for _ in range(n_steps):
            self._pass(vgpu.PASS_PREDICTOR, vgpu.STATE_SPIN)
            self._pass(vgpu.PASS_CORRECTOR, vgpu.STATE_PREDICTOR)
            self._dipole_sum()

    def mc_setup(self, colour: np.ndarray) -> int:
        """Monte Carlo on this shard with the whole system's colouring
        `colour` (one entry per global atom); returns the number of colours."""
        self.ncolours = self.sim.mc_setup(local_colours(colour, self.plan))
        return self.ncolours

    def mc_sweep(self, n_sweeps: int = 1) -> None:
        from . import vgpu
        for _ in range(n_sweeps):
            mc_sweep_sharded(self.ncolours, self.sim.mc_colour, lambda: self._refresh(vgpu.STATE_SPIN))

    def owned_spins(self) -> np.ndarray:
        return self.sim.spins()[:, : self.plan.n_owned]
