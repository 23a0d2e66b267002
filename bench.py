#!/usr/bin/env python3
"""Benchmark of the B200 spin-update hot path.

Workload (one "step" = one stochastic LLG-Heun step of the whole system):
FCC 100^3 unit cells (4,000,000 spins), a=0.354 nm, periodic, two materials
at random 50/50, nearest-neighbour 3x3 tensor exchange (J_AA=J_BB=11.2e-21 J,
J_AB=5e-21 J) plus the reference's three-site DMI with D=0.1 J, cubic
anisotropy Kc=1e-24 J/atom, alpha=0.05, dt=1e-16 s, T=300 K, H=0, spins FP32
SoA with FP64 reductions.  Synthetic, seeded inputs (no dataset is involved).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  value = spin-steps/s over all ranks, timed
on the device with CUDA events on the library's stream between barriers
(max over ranks).  N>1 runs one independent system per GPU (weak scaling,
no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "spin-steps/s on 1 B200 (LLG & MC), batched/adjoint vs plain, % HBM roofline"
PROFILE_EVERY = 10  # timed steps per step whose launches carry CUDA events
UNIT = "spin-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--L", type=int, default=100, help="FCC cells per side (100 = 4M spins)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-dipole", action="store_true", help="leave out the macrocell dipole field")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched and Monte Carlo side results")
    ap.add_argument("--no-error", action="store_true", help="skip the FP32-vs-FP64 error figure of the main line")
    ap.add_argument("--shard", action="store_true",
                    help="strong scaling: one FCC L^3 system cut into N spatial shards (one per GPU), NCCL halo "
                         "exchange of the boundary spins overlapping the core atoms' passes")
    ap.add_argument("--e2e-steps", type=int, default=2000,
                    help="steps of the end-to-end run (the workload's 2,000: initial upload and final download once)")
    ap.add_argument("--records", choices=["auto", "wide"], default="auto",
                    help="bond records: auto = compact words + coupling dictionary when the system allows, "
                         "wide = 16-byte records")
    ap.add_argument("--only", choices=["mc", "batched", "adjoint"], default=None,
                    help="run one side workload alone and print its result (profiling)")
    ap.add_argument("--mc-sweeps", type=int, nargs=2, default=(5000, 10000), metavar=("EQ", "AV"),
                    help="Monte Carlo equilibration and averaging sweeps")
    return ap.parse_args()


def workload_config(L, n_gpus):
    return {"workload": f"FCC {L}^3 LLG-Heun, tensor exchange + 3-site DMI, 2 materials, cubic Kc, T=300K",
            "spins_per_gpu": 4 * L ** 3, "lattice": "fcc", "cells": [L, L, L], "a_nm": 0.354,
            "materials": 2, "exchange": "tensor+DMI (nn, z=12)", "anisotropy": "cubic", "temperature_K": 300.0,
            "dipole": "macrocells 2x2x2 unit cells (125,000 at L=100), tensor solver, update every 100 steps",
            "dt_s": 1e-16, "parallelism": f"replicas x{n_gpus}" if n_gpus > 1 else "single GPU",
            "l2": "inputs larger than L2 (state 96 MB + topology 960 MB per GPU)"}


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region: NVML read every 5 ms from a thread (read-only queries), plus one
    reading at the start and one at the end; nvidia-smi at 200 ms if NVML is
    absent."""
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active")

    def __init__(self, device_index=0, period_s=0.005):
        self.dev = device_index
        self.period = period_s
        self.samples = []  # (sm_mhz, max_mhz, reasons bitmask)
        self.proc = None
        self.nvml = None
        self._stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def _read_nvml(self):
        nv, h = self.nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.samples.append((float(sm), float(mx), int(rs)))

    def _loop(self):
        while not self._stop.is_set():
            try:
                self._read_nvml()
            except Exception:
                return
            time.sleep(self.period)

    def start(self):
        try:
            self.nvml = self._nvml_handle()
            self._read_nvml()
            self.th = threading.Thread(target=self._loop, daemon=True)
            self.th.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.dev), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read_smi, daemon=True)
            self.th.start()
        except FileNotFoundError:
            self.proc = None

    def _read_smi(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            try:
                self.samples.append((float(f[1]), float(f[2]), int(f[4], 16)))
            except (ValueError, IndexError):
                pass

    def stop(self):
        if self.nvml:
            self._stop.set()
            self.th.join(timeout=1.0)
            try:
                self._read_nvml()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return self.summary()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = sorted({nm for _, _, r in self.samples for nm, bit in self.REASONS if r & bit})
        return {"sm_mhz": statistics.median(s[0] for s in self.samples),
                "sm_max_mhz": max(s[1] for s in self.samples), "reasons": reasons,
                "samples": len(self.samples), "source": "nvml 5 ms" if self.nvml else "nvidia-smi 200 ms"}


def measured_peak_hbm():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def traffic_from_profiles(kernel: str, records: str):
    """DRAM bytes per launch of `kernel` ("predictor" / "corrector") with bond
    records `records` ("compact" / "wide") from the committed ncu summary."""
    p = REPO / "profiles" / "ncu_traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get(records, {}).get(kernel)
        except Exception:
            return None
    return None


def byte_model(z=12, b_J=12, multi_mat=True, dipole=False, noise_store=True):
    """Algorithmic HBM bytes per spin per pass (FP32 SoA state, int32 index):
    predictor reads s0 and writes s'; corrector reads s0 and s' and writes s1;
    each pass streams the neighbour words, the per-bond DMI vector (b_J = 12;
    0 with compact records, whose coupling comes from a dictionary of a few
    hundred bytes), the material id and (with the dipole field) the cell id;
    neighbour spins are L2-served.  The thermal Gaussians are generated
    in-register by the predictor; when noise_store it stores the step's
    external field (12 B) for the corrector to read back (12 B) in place of
    the cell id and the field's recomputation; otherwise both passes
    regenerate the noise (0 B)."""
    gather = 4 * (z + 1) + b_J * z + 4 * int(multi_mat) + 4 * int(dipole)
    g = 12 * int(noise_store)
    cell_c = 4 * int(dipole) * int(noise_store)  # the corrector reads no cell id
    return {"predictor": 24 + gather + g, "corrector": 36 + gather + g - cell_c}


def bench_batched(device, steps=2000, plain_steps=200):
    """256 uneven nanoparticles (T ~ U(0,800) K, +2 T -> -2 T sweep) as one
    batch handle in the shape the autotuner picks (the persistent cluster
    kernel replayed as a CUDA graph, or the ordinary step passes over the
    whole batch, cluster 0) against one plain two-launch sequence per
    particle (same kernels)."""
    import torch
    from vampire_b200 import batch as B
    from vampire_b200 import vgpu
    systems, params = B.nanoparticle_ensemble(256)
    n = sum(s.n for s in systems)
    with B.Batch(systems, params, device=device) as b:
        tune = b.autotune(trial_steps=20)
        b.run(100, record_every=100)
        torch.cuda.synchronize()
        stream = torch.cuda.ExternalStream(b_stream(b), device=device)

        def timed(k):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.run(k, record_every=100)
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1)
        ms_b = timed(steps)
        hist = b.history()
        # the best persistent cluster kernel (CUDA graph) beside the pick, when
        # the pick is the ordinary step passes
        persistent = None
        if tune["cluster"] == 0:
            best = None
            for c in (1, 2, 4, 8):
                for bl in (128, 256, 512):
                    try:
                        b.set_shape(c, bl)
                    except Exception:
                        continue
                    b.run(100, record_every=100)
                    ms = timed(100)
                    if best is None or ms < best[0]:
                        best = (ms, c, bl)
            if best:
                b.set_shape(best[1], best[2])
                b.run(100, record_every=100)
                ms_p_best = timed(steps)
                persistent = {"cluster": best[1], "block": best[2], "value": n * steps / (ms_p_best * 1e-3),
                              "ms_per_step": ms_p_best / steps}
    sims = []
    for k, s in enumerate(systems):
        s.params.temperature = params[k]["temperature"]
        sims.append(vgpu.Simulation(s, device=device, noise_seed=k))
    for sim in sims:
        sim.llg_heun(2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for sim in sims:
        sim.llg_heun(plain_steps)
    for sim in sims:
        sim.synchronize()
    ms_p = (time.perf_counter() - t0) * 1e3 * steps / plain_steps
    for sim in sims:
        sim.close()
    mode = "step passes over the whole batch" if tune["cluster"] == 0 else "persistent cluster kernel, CUDA graph"
    return {"systems": 256, "spins": n, "steps": steps, "shape": tune, "mode": mode, "persistent_graph": persistent,
            "value": n * steps / (ms_b * 1e-3), "unit": UNIT, "ms": ms_b,
            "plain_per_system_value": n * steps / (ms_p * 1e-3), "speedup_vs_per_system": ms_p / ms_b,
            "records": int(hist.shape[0]),
            "timing": "batch: CUDA events on the batch stream; per-system: host wall clock of 256 "
                      f"launch sequences of {plain_steps} steps, scaled to {steps}"}


def b_stream(b):
    import ctypes as C
    from vampire_b200 import vgpu
    p = C.c_void_p()
    vgpu.check(vgpu.lib().vgpu_get_stream(b.handle, C.byref(p)), b.handle)
    return p.value


def _tc_fit(T, m):
    """Curie temperature from <|m|>(T) ~ a (1 - T/Tc)^b (points with m > 0.3)."""
    import numpy as np
    from scipy.optimize import curve_fit
    sel = (m > 0.3) & (T > 0)
    f = lambda t, tc, b, a: a * np.clip(1 - t / tc, 1e-12, None) ** b
    p, _ = curve_fit(f, T[sel], m[sel], p0=(1.05 * T[sel].max(), 0.35, 1.0), maxfev=20000)
    return float(p[0])


def bench_mc(device, L=50, eq=5000, av=10000, every=10):
    """The Curie-sweep protocol on SC 50^3 (125,000 spins, J, Ku and mu_s of
    the SC ferromagnet, H = 0): 31 temperatures 0..1500 K as replicas of one
    handle (3,875,000 spins), checkerboard Metropolis with angle moves,
    `eq` equilibration then `av` averaging sweeps, device-side running means
    of <|m|> per replica every `every` sweeps.  Timed with CUDA events over
    the whole protocol (sweeps and statistics)."""
    import numpy as np
    import torch
    from vampire_b200 import system as S
    from vampire_b200 import vgpu
    base = S.config_sc_llg(L, temperature=0.0)
    base.params.H_applied = 0.0
    base.spins = np.tile(np.array([[0.0], [0.0], [1.0]]), (1, base.n))
    Ts = np.arange(0.0, 1501.0, 50.0)
    s = S.replicas(base, Ts)
    with vgpu.Simulation(s, device=device, noise_seed=4242) as sim:
        mid = sim.add_mask(*s.masks["replica"])
        nc = sim.mc_setup()
        stream = torch.cuda.ExternalStream(sim.stream_ptr(), device=device)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        sim.synchronize()
        e0.record(stream)
        sim.mc_sweep(eq)
        e1.record(stream)
        sim.stats_reset()
        for _ in range(av // every):
            sim.mc_sweep(every)
            sim.stats_update(magnetization=True)
        e2.record(stream)
        e2.synchronize()
        ms = e0.elapsed_time(e2)
        ms_eq = e0.elapsed_time(e1)
        _, mean, cnt = sim.magnetization(mid)
        moves, rej = sim.mc_counters()
    m_T = mean.reshape(-1, 4)[:, 3] / max(cnt, 1)
    try:
        tc = _tc_fit(Ts, m_T)
    except Exception:
        tc = None
    sweeps = eq + (av // every) * every
    return {"workload": f"SC {L}^3 x {Ts.size} temperatures {Ts[0]:g}-{Ts[-1]:g} K (replicas in one handle), "
                        f"{eq} + {av} sweeps, <|m|> every {every} sweeps",
            "spins": s.n, "colours": nc, "sweeps": sweeps, "value": s.n * sweeps / (ms * 1e-3),
            "unit": "spin-moves/s", "sweep_only_value": s.n * eq / (ms_eq * 1e-3), "protocol_s": ms * 1e-3,
            "acceptance": 1.0 - rej / moves, "Tc_K": tc, "m_T": [round(float(x), 5) for x in m_T],
            "error_vs_reference": mc_reference_comparison(Ts, m_T, tc, (eq, av, every))}


def bench_adjoint(device, L=32, steps=2000):
    """Adjoint LLG-Heun on SC 32^3 (32,768 spins), T=0, 2,000 steps: the
    gradient of the trajectory loss w.r.t. (J, Ku, H) at J=11.2e-21 J,
    Ku=6.69e-24 J, H=(0,0,0.4) T against the target m_z(t) of J=10e-21 J,
    Ku=5e-24 J, H=(0,0,0.5) T; the FP32 production build (FP64 sums for m_z,
    the loss and the gradients), sqrt(N) checkpointing, with the FP64 debug
    build timed beside it.  Timed around AdjointRunner.loss_and_grad: the
    system set-up and upload and the C-ABI call (forward with checkpoints,
    segment recomputation and the backward sweep); the median of five calls
    after two warm-up calls."""
    from vampire_b200 import adjoint as A
    run = A.AdjointRunner(L=L, device=device, precision="fp32")
    run64 = A.AdjointRunner(L=L, device=device, precision="fp64")
    target = run64.trajectory(10e-21, 5e-24, (0.0, 0.0, 0.5), steps)
    for _ in range(2):  # warm-up (module loading, first allocations)
        run.loss_and_grad(11.2e-21, 6.69e-24, (0.0, 0.0, 0.4), target)
    # five timed gradients, the median reported: the host wall clock around
    # ~20,000 launches varies between runs on a shared host
    times = []
    for _ in range(5):
        t0 = time.perf_counter()
        loss, grad = run.loss_and_grad(11.2e-21, 6.69e-24, (0.0, 0.0, 0.4), target)
        times.append(time.perf_counter() - t0)
    dt = sorted(times)[2]
    run64.loss_and_grad(11.2e-21, 6.69e-24, (0.0, 0.0, 0.4), target)  # warm-up
    times64 = []
    for _ in range(5):
        t0 = time.perf_counter()
        loss64, grad64 = run64.loss_and_grad(11.2e-21, 6.69e-24, (0.0, 0.0, 0.4), target)
        times64.append(time.perf_counter() - t0)
    # error: the adjoint gradient against central differences (h = 1e-6
    # relative) of the device FP64 forward loss, for J, Ku and H_z
    import numpy as np
    p = np.array([11.2e-21, 6.69e-24, 0.0, 0.0, 0.4])
    rel = []
    for k, sc in ((0, p[0]), (1, p[1]), (4, 0.4)):
        h = 1e-6 * sc
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (run64.loss_and_grad(pp[0], pp[1], pp[2:], target)[0] -
              run64.loss_and_grad(pm[0], pm[1], pm[2:], target)[0]) / (2 * h)
        rel.append(abs(grad[k] - fd) / abs(fd))
    return {"workload": f"SC {L}^3, {steps} steps, loss = sum_t dt (m_z - target)^2, grad w.r.t. J, Ku, H (3)",
            "spins": L ** 3, "steps": steps, "seconds": dt, "seconds_all": times, "value": L ** 3 * steps / dt,
            "unit": "spin-steps/s (forward + backward)", "precision": "fp32",
            "fp64_build": {"seconds": sorted(times64)[2], "value": L ** 3 * steps / sorted(times64)[2],
                           "max_rel_grad_dev_fp32": float(np.max(np.abs(grad - grad64)[[0, 1, 4]] /
                                                                 np.abs(grad64)[[0, 1, 4]]))},
            "loss": loss,
            "grad": [float(g) for g in grad], "checkpoints": int(-(-steps // int(steps ** 0.5 + 0.999999))),
            "error_vs_fd": {"max_rel_dev": float(max(rel)), "components": ["J", "Ku", "Hz"],
                            "against": "central differences (h = 1e-6 relative) of the FP64 forward loss"}}


def error_vs_fp64_llg(sysm, device, steps=100):
    """Max per-spin component deviation of the FP32 passes from the FP64 build
    of the same kernels (which follows the reference's own trajectories to
    1e-12 in the tests) on the workload system at T = 0 -- deterministic, so
    the two runs see the same dynamics -- over the first `steps` steps, the
    dipole field included."""
    import numpy as np
    from vampire_b200 import vgpu
    T0 = sysm.params.temperature
    sysm.params.temperature = 0.0
    out = {}
    try:
        for prec in ("fp32", "fp64"):
            with vgpu.Simulation(sysm, device=device, precision=prec) as sim:
                if sysm.cells is not None:
                    sim.dipole_setup(sysm.cells)
                sim.llg_heun(steps)
                out[prec] = sim.spins()
    finally:
        sysm.params.temperature = T0
    return {"max_abs_spin_dev": float(np.abs(out["fp32"] - out["fp64"]).max()), "steps": steps,
            "against": "FP64 build of the same kernels, same system at T=0 (FP32 bound 1e-5 over 100 steps)"}


def error_vs_fp64_batched(device, steps=100, n_plain=16):
    """The batched ensemble at T = 0 with every spin tilted at random from
    the saturated start (so that the dynamics is not the fixed point of a
    field along the magnetisation): max per-spin deviation after `steps` of
    the FP32 batch, in the step-pass shape and in a persistent shape, from
    the FP64 batch, and of FP32 per-system launches from FP64 ones (the first
    n_plain particles)."""
    import numpy as np
    from vampire_b200 import batch as B
    from vampire_b200 import vgpu
    systems, params = B.nanoparticle_ensemble(256, temperature=0.0)
    rng = np.random.default_rng(1)
    for s in systems:
        sp = s.spins + 0.4 * rng.standard_normal(s.spins.shape)
        s.spins = sp / np.linalg.norm(sp, axis=0)
    got = {}
    for key, prec, shape in (("fp64", "fp64", (1, 256)), ("passes", "fp32", (0, 0)),
                             ("persistent", "fp32", (8, 128))):
        with B.Batch(systems, params, device=device, precision=prec) as b:
            b.set_shape(*shape)
            b.run(steps, record_every=0)
            got[key] = b.spins()
    dev = {k: max(float(np.abs(a - c).max()) for a, c in zip(got[k], got["fp64"])) for k in ("passes", "persistent")}
    dev_p = 0.0
    for k in range(n_plain):
        s = systems[k]
        s.params.temperature = 0.0
        r = {}
        for prec in ("fp32", "fp64"):
            with vgpu.Simulation(s, device=device, precision=prec) as sim:
                sim.llg_heun(steps)
                r[prec] = sim.spins()
        dev_p = max(dev_p, float(np.abs(r["fp32"] - r["fp64"]).max()))
    return {"batched_max_abs_spin_dev": dev["passes"], "persistent_max_abs_spin_dev": dev["persistent"],
            "per_system_max_abs_spin_dev": dev_p, "steps": steps,
            "against": f"FP64 batch at T=0 from tilted spins (batched: all 256, step passes and persistent "
                       f"cluster 8 x 128; per-system launches: first {n_plain})"}


def mc_reference_comparison(T, m_T, tc, sweeps):
    """The Monte Carlo m(T) against the reference's own sequential sweep of
    the same protocol (tests/golden/mc_sc50_curie.npz, made by the reference
    program), when that fixture is present and the temperatures and sweep
    counts (equilibration, averaging, sampling interval) are the fixture's."""
    import numpy as np
    p = REPO / "tests" / "golden" / "mc_sc50_curie.npz"
    if not p.exists():
        return None
    d = np.load(p)
    if not np.array_equal(d["T"], T) or tuple(int(x) for x in d["sweeps"]) != tuple(sweeps):
        return None
    ref = d["m_mean"]
    try:
        tc_ref = _tc_fit(T, ref)
    except Exception:
        tc_ref = None
    return {"max_abs_m_dev": float(np.abs(np.asarray(m_T) - ref).max()), "Tc_ref_K": tc_ref,
            "Tc_rel_dev": (abs(tc - tc_ref) / tc_ref) if (tc and tc_ref) else None,
            "against": "reference sequential Metropolis, SC 50^3, same temperatures and sweeps"}


def reference_sample_L(steps, budget_s=20.0, rate_per_proc=3.0e6):
    """FCC cells per side of the reference arm's sample: the largest of 50,
    40, 30, 20 whose `steps` timed steps take about `budget_s` or less at
    `rate_per_proc` spin-steps/s per process (the reference's FCC tensor rate
    with all cores busy), so the arm stays within a few minutes at any step
    count while its timed region lasts seconds."""
    for L in (50, 40, 30, 20):
        if steps * 4 * L ** 3 / rate_per_proc <= budget_s:
            return L
    return 20


def reference_arm(args, rank, world):
    if rank != 0:
        return
    from oracle import cpu_baseline as B
    procs = os.cpu_count() or 1
    # each step: one Heun step of an FCC L^3 sample (no dipole field: the
    # reference's dense cell tensor does not fit at the workload's 125,000
    # cells) in every process; W untimed steps, then exactly K timed ones
    steps, warmup = args.steps, args.warmup
    L = reference_sample_L(steps)
    try:
        r = B.reference_rate(L=L, steps=steps, procs=procs, warmup=warmup)
    except Exception as e:  # binary absent: fall back to the restatement
        try:
            r = B.port_rate(L=16, steps=20)
        except Exception as e2:
            print(json.dumps({"impl": "reference", "unavailable": f"{e}; {e2}"}))
            return
    cfg = {"workload": f"FCC {L}^3 LLG-Heun, tensor exchange + 3-site DMI, 2 materials, cubic Kc, T=300K, "
                       "no dipole field", "spins_per_process": 4 * L ** 3, "processes": r["cores"],
           "lattice": "fcc", "cells": [L, L, L], "a_nm": 0.354, "materials": 2, "exchange": "tensor+DMI (nn, z=12)",
           "anisotropy": "cubic", "temperature_K": 300.0, "dipole": "off", "dt_s": 1e-16,
           "stands_for": "the FCC 100^3 workload (4,000,000 spins, dipole on) of the GPU arm: spin-steps/s is an "
                         "intensive rate, so a bounded sample of the same physics is timed per process",
           "parallelism": f"{r['cores']} independent reference processes (the reference is single-threaded)"}
    # n_gpus: the N this arm was launched for (it runs on the host cores alone)
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": r.get("ms_per_step"), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "timed_region_s": (r.get("ms_per_step") or 0.0) * steps * 1e-3,
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def shard_arm(args, rank, world, local, dist):
    """--shard: the workload system (FCC L^3, dipole field on) cut into
    `world` spatial shards of equal atom count (vampire_b200.shard), one per
    GPU: each pass exchanges its input state's halo over NCCL on a
    communication stream while the core atoms run, then runs the boundary
    atoms; the dipole cell moments are all-reduced every 100 steps.  Strong
    scaling: value = all spins x steps / the slowest rank's CUDA-event time."""
    import torch
    from vampire_b200 import shard as SH
    from vampire_b200 import system as S
    sysm = S.config_fcc_tensor(L=args.L, seed=2024, dipole=not args.no_dipole)
    plan = SH.make_plan(sysm, world)[rank]
    sh = SH.ShardedSimulation(sysm, plan, device=local, precision="fp32", noise_seed=1000)
    if sysm.cells is not None:
        sh.dipole_setup(sysm.cells)
    sh.step(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(sh.stream)
    sh.step(args.steps)
    ev1.record(sh.stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    if dist:
        tt = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = sysm.n * args.steps / (ms * 1e-3)
    if rank == 0:
        cfg = workload_config(args.L, world)
        cfg["parallelism"] = (f"{world} spatial shards (index slabs), NCCL halo exchange overlapping the core atoms"
                              if world > 1 else "one shard (no exchange)")
        cfg["ranges"] = {"core": list(sh.ranges[0]) if sh.ranges else None, "owned": plan.n_owned,
                         "halo": int(plan.halo.size)}
        print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                          "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                          "config": cfg, "clocks": clk, "mode": "shard", "e2e": None,
                          "gpu_launches": None}), flush=True)
    sh.sim.close()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.shard:
        from vampire_b200 import build as vbuild
        vbuild.build()
        torch.cuda.set_device(local)
        shard_arm(args, rank, world, local, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.only:
        from vampire_b200 import build as vbuild
        vbuild.build()
        torch.cuda.set_device(local)
        fn = {"mc": lambda: bench_mc(local, eq=args.mc_sweeps[0], av=args.mc_sweeps[1]),
              "batched": lambda: bench_batched(local), "adjoint": lambda: bench_adjoint(local)}[args.only]
        r = fn()
        if rank == 0:
            print(json.dumps({"only": args.only, **{k: v for k, v in r.items() if k != "m_T"}}), flush=True)
        if dist:
            dist.destroy_process_group()
        return

    from vampire_b200 import build as vbuild
    from vampire_b200 import system as S
    from vampire_b200 import vgpu
    vbuild.build()
    torch.cuda.set_device(local)
    sysm = S.config_fcc_tensor(L=args.L, seed=2024 + rank, dipole=not args.no_dipole)
    sim = vgpu.Simulation(sysm, device=local, precision="fp32", noise_seed=1000 + rank)
    if args.records == "wide":
        sim.set_option(vgpu.OPT_COMPACT_RECORDS, 0)
    layout, ndict = sim.record_layout()
    if sysm.cells is not None:
        sim.dipole_setup(sysm.cells)
    mask_id = sim.add_mask(*sysm.masks["system"])
    stream = torch.cuda.ExternalStream(sim.stream_ptr(), device=local)

    # warm-up
    sim.llg_heun(args.warmup)
    sim.synchronize()
    # the dipole field update (every 100 steps): timed alone here so that its
    # share enters `value` whatever the timed window holds
    upd_ms, rate = 0.0, 0
    if sysm.cells is not None:
        rate = int(sysm.cells.get("update_rate", 100))
        u0, u1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sim.dipole_update()
        sim.synchronize()
        u0.record(stream)
        for _ in range(3):
            sim.dipole_update()
        u1.record(stream)
        u1.synchronize()
        upd_ms = u0.elapsed_time(u1) / 3
    step0 = sim.step

    def barrier():
        if dist:
            dist.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    sim.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    # per-launch CUDA events on the launches of one step in `every` of the
    # timed region (events between every pair of launches would slow the
    # stream itself); at least 4 sampled launches per pass
    every = max(1, min(PROFILE_EVERY, args.steps // 4))
    sim.set_option(vgpu.OPT_PROFILE_EVERY, every)
    sim.profile(True)
    ev0.record(stream)
    sim.llg_heun(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    sim.synchronize()
    torch.cuda.synchronize()
    barrier()
    prof = sim.profile_read()
    sim.profile(False)
    clk = clocks.stop()
    ms_window = ev0.elapsed_time(ev1)
    # updates that fell inside the window (after the step that brings the
    # counter to a multiple of the rate) against the steps' share of them
    k_in = (step0 + args.steps) // rate - step0 // rate if rate else 0
    ms = ms_window + ((args.steps / rate - k_in) * upd_ms if rate else 0.0)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    n = sysm.n
    value = n * args.steps * world / (ms * 1e-3)

    # --- roofline of the dominant kernel --------------------------------
    compact = layout in (vgpu.RECORDS_COMPACT, vgpu.RECORDS_WINDOW)
    bm = byte_model(b_J=0 if compact else 12, dipole=sysm.cells is not None)
    records = (f"compact: 4 B per bond (neighbour | coupling index) + {ndict}-entry coupling dictionary"
               if compact else "16 B per bond (neighbour, DMI vector)")
    if layout == vgpu.RECORDS_WINDOW:
        records += "; neighbour spins staged per tile in shared memory (window staging)"
    kern = max(("predictor", "corrector"), key=lambda k: prof[k]["ms"])
    avg_ms = prof[kern]["ms"] / max(1, prof[kern]["count"])
    peak, peak_kind = measured_peak_hbm()
    achieved = bm[kern] * n / (avg_ms * 1e-3) / 1e9
    traffic = traffic_from_profiles(kern, "compact" if compact else "wide")
    step_gbs = (bm["predictor"] + bm["corrector"]) * n * args.steps / (ms * 1e-3) / 1e9

    # --- e2e through the C ABI with host buffers ------------------------
    e2e = None
    if not args.no_e2e:
        import numpy as np
        # pinned host buffers: the copies are DMAs straight from/to them
        host_in = torch.from_numpy(np.ascontiguousarray(sysm.spins)).pin_memory()
        host_out = torch.empty((3, n), dtype=torch.float64).pin_memory()
        host_spins, final_buf = host_in.numpy(), host_out.numpy()
        K = args.e2e_steps
        # per step: the step's input (applied field of a slow sweep, passed
        # to the passes as kernel arguments), one step, the statistics, and
        # a read-back of the step's magnetisation into pinned host memory;
        # step t's read-back is waited for while step t+1 runs
        rows = [torch.zeros(9 * sysm.masks["system"][1], dtype=torch.float64).pin_memory() for _ in range(2)]
        evs = [torch.cuda.Event() for _ in range(2)]
        p = sysm.params
        p0 = p.H_applied
        barrier()
        sim.synchronize()
        t0 = time.perf_counter()
        sim.set_spins(host_spins)                 # H2D: initial spins from host
        m_trace = []
        for t in range(K):
            p.H_applied = p0 + 1e-3 * t / K       # the step's input
            sim.set_params(p)
            sim.llg_heun(1)
            sim.stats_update(magnetization=True)
            sim.stats_copy_rows(mask_id, rows[t % 2].data_ptr())   # D2H: the step's result
            evs[t % 2].record(stream)
            if t > 0:
                evs[(t - 1) % 2].synchronize()
                m_trace.append(float(rows[(t - 1) % 2][3]))
        evs[(K - 1) % 2].synchronize()
        m_trace.append(float(rows[(K - 1) % 2][3]))
        final = sim.spins(out=final_buf)          # D2H: final spins to host
        t1 = time.perf_counter()
        p.H_applied = p0
        sim.set_params(p)
        e2e_s = t1 - t0
        if dist:
            t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        h2d = (3 * n * 8) / K + 64
        d2h = 9 * 8 * sysm.masks["system"][1] + (3 * n * 8) / K
        e2e = {"value": n * K * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": K,
               "path": "vgpu_set_spins from pinned host FP64; per step vgpu_set_params (applied-field sweep) + "
                       "vgpu_llg_heun(1) + vgpu_stats_update + vgpu_stats_copy_rows into pinned host memory, "
                       "read on the host one step later; then vgpu_get_spins into pinned host FP64"}
        assert len(m_trace) == K and np.isfinite(m_trace).all()
        assert np.isfinite(final).all()

    extra = {}
    sim.close()
    err = None
    if not args.no_error:
        err = error_vs_fp64_llg(sysm, local)
    if not args.no_extras:
        extra["batched"] = bench_batched(local)
        extra["batched"]["error_vs_fp64"] = error_vs_fp64_batched(local)
        extra["monte_carlo"] = bench_mc(local, eq=args.mc_sweeps[0], av=args.mc_sweeps[1])
        extra["adjoint"] = bench_adjoint(local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import cpu_baseline as B
            cpu = B.best_available(L=40, steps=150, procs=1)
            cpu.pop("wall_s", None)
        except Exception as e:
            cpu = {"value": None, "unavailable": str(e)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.L, world),
            "roofline": {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_spin": bm, "bond_records": records,
                         "avg_launch_ms": {k: prof[k]["ms"] / max(1, prof[k]["count"])
                                           for k in ("predictor", "corrector")},
                         "timed_launches": {k: prof[k]["count"] for k in ("predictor", "corrector")},
                         "launch_timing": f"CUDA events around the launches of one step in {every} "
                                          "of the timed region",
                         "step_achieved_gbs": step_gbs},
            "dipole_update": {"ms": upd_ms, "every_steps": rate, "updates_in_window": k_in,
                              "amortised_ms_per_step": (upd_ms / rate if rate else 0.0),
                              "window_ms": ms_window,
                              "note": "ms_per_step = (window + (steps/rate - updates_in_window) x update ms) / steps"},
            "error_vs_fp64": err,
            "gpu_launches": prof["kernel_launches"],
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
