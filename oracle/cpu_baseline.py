"""CPU baselines for bench.py (test/measurement infrastructure only).

* ``reference``: the reference program's own CPU LLG-Heun
  (sim::LLG_Heun, src/simulate/LLGHeun.cpp:160-282) run through
  oracle/_ref/vampire-harness on a bounded sample of the benchmark workload:
  FCC L^3 periodic, two-material random A/B alloy, nn tensor exchange with the
  three-site DMI, cubic anisotropy, T=300 K.  The reference is
  single-threaded, so all host cores are used by running one independent
  process per core; the rate is the sum of spins*steps over the slowest
  process's step-loop time (the harness times its own loop, excluding setup).
* ``port``: the FP64 C restatement (oracle/vref.c) on the same kind of
  sample, one thread -- used only when the reference binary is absent.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

from . import oracle as O
from .refinputs import fcc_input, fcc_mat


def _one_reference(L: int, steps: int, T: float, warmup: int = 0) -> tuple:
    tmp = tempfile.mkdtemp(prefix="vref_bench_")
    Path(tmp, "input").write_text(fcc_input(L, T=T))
    Path(tmp, "m.mat").write_text(fcc_mat())
    out = Path(tmp, "out")
    out.mkdir()
    r = subprocess.run([str(O.HARNESS), "--out", str(out), "--steps", str(steps), "--warmup", str(warmup), "--time"],
                       cwd=tmp,
                       capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(f"reference harness failed: {r.stdout[-500:]} {r.stderr[-500:]}")
    for line in r.stdout.splitlines():
        if line.startswith("HARNESS_LOOP_SECONDS"):
            f = line.split()
            return float(f[1]), int(f[3]), int(f[5])
    raise RuntimeError("harness printed no loop time")


def reference_rate(L: int = 20, steps: int = 100, procs: int = 0, T: float = 300.0, warmup: int = 0) -> dict:
    """Aggregate spin-steps/s of `procs` concurrent reference processes."""
    if not O.harness_available():
        raise FileNotFoundError("oracle/_ref/vampire-harness not built")
    procs = procs or (os.cpu_count() or 1)
    wall0 = time.time()
    with ThreadPoolExecutor(procs) as ex:
        res = list(ex.map(lambda _: _one_reference(L, steps, T, warmup), range(procs)))
    loop = max(r[0] for r in res)
    atoms = res[0][1]
    total = sum(r[1] * r[2] for r in res)
    return {"value": total / loop, "unit": "spin-steps/s", "cores": procs, "kind": "reference",
            "sample": f"{procs} x reference vampire LLG-Heun (sim::LLG_Heun), FCC {L}^3 periodic "
                      f"({atoms} spins), A/B alloy, tensor exchange + DMI + cubic, T={T:g} K, {warmup} untimed + {steps} timed steps "
                      f"each; step-loop time of the slowest process",
            "wall_s": time.time() - wall0, "ms_per_step": loop / steps * 1e3}


def port_rate(L: int = 20, steps: int = 50, T: float = 300.0) -> dict:
    """Single-thread FP64 restatement (oracle/vref.c) on the same sample shape."""
    from vampire_b200 import system as S
    s = S.config_fcc_tensor(L=L, temperature=T)
    o = O.OracleSystem(s)
    rng = np.random.default_rng(0)
    xi = rng.standard_normal(3 * s.n * steps)
    t0 = time.perf_counter()
    o.llg_heun(s.spins, steps, xi=xi)
    dt = time.perf_counter() - t0
    return {"value": s.n * steps / dt, "unit": "spin-steps/s", "cores": 1, "kind": "port",
            "sample": f"FP64 C restatement of sim::LLG_Heun, FCC {L}^3 ({s.n} spins), tensor+DMI+cubic, "
                      f"T={T:g} K, {steps} steps, 1 thread"}


def best_available(L: int = 20, steps: int = 100, procs: int = 1) -> dict:
    try:
        return reference_rate(L, steps, procs)
    except (FileNotFoundError, RuntimeError, OSError):
        return port_rate(L, max(10, steps // 2))
