"""Batched independent systems: builder for the nanoparticle ensemble and a
wrapper of the vgpu_batch_* C ABI (include/vgpu.h).

The ensemble: simple-cubic spheres (a = 0.3 nm, open boundaries) with
diameters drawn lognormal (median 4 nm, sigma 0.3 of ln d, clipped to
2-8 nm), the material of the simple-cubic benchmark (J = 11.2e-21 J,
Ku = 6.69e-24 J along z, mu_s = 1.72 muB, alpha = 0.1), each particle with
its own temperature drawn uniform in 0-800 K and its own applied field swept
linearly from +2 T to -2 T along z (a hysteresis loop).
"""
from __future__ import annotations

import ctypes as C
import json
import os
from pathlib import Path
from typing import List, Optional, Sequence

import numpy as np

from . import system as S
from . import vgpu as V


class BatchSystemC(C.Structure):
    _fields_ = [("temperature", C.c_double), ("H_start", C.c_double * 3), ("H_end", C.c_double * 3),
                ("n_ramp", C.c_uint64)]


def sphere(diameter_nm: float, a: float = 3.0, material: Optional[S.Material] = None,
           params: Optional[S.SimParams] = None, spin_seed: int = 0) -> S.SpinSystem:
    """Simple-cubic sphere of the given diameter (open boundaries)."""
    d = diameter_nm * 10.0
    L = int(np.ceil(d / a)) + 1
    c = (L - 1) * a / 2.0
    g = np.arange(L) * a - c
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    keep = (x * x + y * y + z * z <= (d / 2.0) ** 2).ravel()
    m = material or S.Material(alpha=0.1, mu_s_muB=1.72, Ku=6.69e-24)
    p = params or S.SimParams(dt_SI=1e-16)
    return S.build("sc", L, L, L, a, [m], [[11.2e-21]], p, periodic=(False, False, False), keep=keep,
                   spin_seed=spin_seed)


def nanoparticle_ensemble(n: int = 256, seed: int = 7, n_ramp: int = 20000, t_max: float = 800.0,
                          temperature: Optional[float] = None):
    """(systems, per-system parameters) of the batched benchmark ensemble."""
    rng = np.random.default_rng(seed)
    diam = np.clip(np.exp(np.log(4.0) + 0.3 * rng.standard_normal(n)), 2.0, 8.0)
    temps = rng.uniform(0.0, t_max, n) if temperature is None else np.full(n, float(temperature))
    systems, params = [], []
    for k in range(n):
        s = sphere(float(diam[k]), spin_seed=seed * 1000 + k)
        # start saturated along +z (the top of the hysteresis loop)
        s.spins = np.tile(np.array([[0.0], [0.0], [1.0]]), (1, s.n))
        systems.append(s)
        params.append({"temperature": float(temps[k]), "H_start": (0.0, 0.0, 2.0), "H_end": (0.0, 0.0, -2.0),
                       "n_ramp": int(n_ramp)})
    return systems, params


class Batch:
    """All systems of a batch resident on one GPU (one vgpu handle)."""

    def __init__(self, systems: Sequence[S.SpinSystem], params: Sequence[dict], device: int = 0,
                 precision: str = "fp32", noise_seed: int = 0, common: Optional[S.SimParams] = None):
        self.systems = list(systems)
        self.n_sys = len(self.systems)
        keep = []
        descs = (V.SystemDesc * self.n_sys)()
        for k, s in enumerate(self.systems):
            d, kk = V._desc(s)
            descs[k] = d
            keep.append(kk)
        bs = (BatchSystemC * self.n_sys)()
        for k, p in enumerate(params):
            bs[k].temperature = p["temperature"]
            for c in range(3):
                bs[k].H_start[c] = p["H_start"][c]
                bs[k].H_end[c] = p["H_end"][c]
            bs[k].n_ramp = int(p.get("n_ramp", 0))
        # an empty batch reaches the library, which refuses it (VGPU_ERR_ARG)
        cp = V.params_struct(common or (self.systems[0].params if self.systems else S.SimParams()))
        self._h = C.c_void_p()
        prec = V.PREC_FP64 if precision == "fp64" else V.PREC_FP32
        V.check(V.lib().vgpu_batch_create(device, prec, C.c_int32(self.n_sys), descs, bs, C.byref(cp),
                                          C.byref(self._h)))
        self._check(V.lib().vgpu_set_noise(self._h, C.c_int(V.NOISE_PHILOX), C.c_uint64(noise_seed)))
        self.ranges = []
        for k in range(self.n_sys):
            f, m = C.c_int32(), C.c_int32()
            self._check(V.lib().vgpu_batch_system_range(self._h, C.c_int32(k), C.byref(f), C.byref(m)))
            self.ranges.append((f.value, m.value))
        self.n = sum(m for _, m in self.ranges)

    def _check(self, rc):
        V.check(rc, self._h)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            V.lib().vgpu_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_shape(self, cluster: int, block: int) -> None:
        self._check(V.lib().vgpu_batch_set_shape(self._h, C.c_int32(cluster), C.c_int32(block)))

    def autotune(self, trial_steps: int = 50, cache: Optional[Path] = None):
        """Pick cluster size and block size by timing them on this batch;
        results are cached per (systems, atoms, device) in `cache` (JSON)."""
        key = f"{self.n_sys}:{self.n}"
        if cache is not None and cache.exists():
            try:
                got = json.loads(cache.read_text()).get(key)
                if got:
                    self.set_shape(got["cluster"], got["block"])
                    return got
            except (ValueError, V.VGPUError):
                pass
        c, b, ms = C.c_int32(), C.c_int32(), C.c_double()
        self._check(V.lib().vgpu_batch_autotune(self._h, C.c_int32(trial_steps), C.byref(c), C.byref(b),
                                                 C.byref(ms)))
        got = {"cluster": c.value, "block": b.value, "ms_per_step": ms.value}
        if cache is not None:
            data = {}
            if cache.exists():
                try:
                    data = json.loads(cache.read_text())
                except ValueError:
                    data = {}
            data[key] = got
            cache.parent.mkdir(parents=True, exist_ok=True)
            cache.write_text(json.dumps(data, indent=1))
        return got

    def run(self, n_steps: int, record_every: int = 0, graph: bool = True) -> None:
        self._check(V.lib().vgpu_batch_run(self._h, C.c_uint64(n_steps), C.c_uint32(record_every),
                                           C.c_int32(int(graph))))

    def llg_heun(self, n_steps: int = 1) -> None:
        """Two plain launches per step over the whole batch."""
        self._check(V.lib().vgpu_llg_heun(self._h, C.c_uint64(n_steps)))

    def history(self) -> np.ndarray:
        n = C.c_int64()
        self._check(V.lib().vgpu_batch_history(self._h, C.cast(None, C.POINTER(C.c_double)), C.c_int64(0),
                                               C.byref(n)))
        out = np.empty(max(1, n.value) * self.n_sys * 4)
        self._check(V.lib().vgpu_batch_history(self._h, out.ctypes.data_as(C.POINTER(C.c_double)),
                                               C.c_int64(n.value), C.byref(n)))
        return out[: n.value * self.n_sys * 4].reshape(n.value, self.n_sys, 4)

    def spins(self) -> List[np.ndarray]:
        out = np.empty((3, self.n))
        p = [out[q].ctypes.data_as(C.POINTER(C.c_double)) for q in range(3)]
        self._check(V.lib().vgpu_get_spins(self._h, *p))
        return [out[:, f:f + m] for f, m in self.ranges]

    @property
    def step(self) -> int:
        v = C.c_uint64()
        self._check(V.lib().vgpu_get_step(self._h, C.byref(v)))
        return v.value

    def profile(self, enable: bool) -> None:
        self._check(V.lib().vgpu_profile(self._h, C.c_int(int(enable))))
