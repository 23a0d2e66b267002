"""Spin snapshots in the reference's configuration-output formats.

The reference writes, every configuration output step, the spins of its
output atoms (src/config/atoms_spins.cpp): a data file "spins-%08d.data" --
binary: a uint64 atom count, then x, y, z of every output atom as FP64
(src/config/write.cpp:107-140); text: the count on a line, then one
tab-separated line per atom (write.cpp:62-95) -- and a meta file
"spins-%08d.meta" with the time, field, temperature and magnetisation
(src/config/meta.cpp:98-140).  The output atoms are those inside the output
bounds, fractions of the system size (src/config/initialize.cpp:28-55).

Here the gather of the output atoms' spins into the file's data block runs on
the device (`Simulation.snapshot`, vgpu_snapshot); this module lists the
output atoms and writes the files byte for byte as the reference does.
"""
from __future__ import annotations

import time
from pathlib import Path
from typing import Optional, Sequence

import numpy as np


def output_atom_list(coords: np.ndarray, system_dimensions: Sequence[float],
                     minimum: Sequence[float] = (0.0, 0.0, 0.0),
                     maximum: Sequence[float] = (1.0, 1.0, 1.0)) -> np.ndarray:
    """Ids of the atoms inside the output bounds, in atom order: coordinate c
    of every axis within [minimum * dimension, maximum * dimension]
    (config::internal::initialize, src/config/initialize.cpp:28-55).
    coords: (3, n) in the units of system_dimensions."""
    lo = np.asarray(minimum, dtype=np.float64) * np.asarray(system_dimensions, dtype=np.float64)
    hi = np.asarray(maximum, dtype=np.float64) * np.asarray(system_dimensions, dtype=np.float64)
    inside = np.ones(coords.shape[1], dtype=bool)
    for ax in range(3):
        inside &= (coords[ax] >= lo[ax]) & (coords[ax] <= hi[ax])
    return np.flatnonzero(inside).astype(np.int64)


def _g(x: float) -> str:
    # std::ostream's default floating-point output: %g, 6 significant digits
    return "%g" % x


def write_spins_binary(path, data: np.ndarray) -> None:
    """Binary spin file: uint64 count, then the (3 count) FP64 data block."""
    data = np.ascontiguousarray(data, dtype=np.float64)
    with open(path, "wb") as f:
        f.write(np.array([data.size // 3], dtype=np.uint64).tobytes())
        f.write(data.tobytes())


def write_spins_text(path, data: np.ndarray) -> None:
    """Text spin file: the count, then x<TAB>y<TAB>z per atom (%g)."""
    d = np.asarray(data, dtype=np.float64).reshape(-1, 3)
    with open(path, "w") as f:
        f.write(f"{d.shape[0]}\n")
        f.writelines(f"{_g(x)}\t{_g(y)}\t{_g(z)}\n" for x, y, z in d)


def write_spins_meta(path, data_name: str, time_s: float, temperature: float, field_unit: Sequence[float],
                     field_strength: float, magnetization: Sequence[float], date: Optional[str] = None) -> None:
    """Meta file of one snapshot (config::internal::write_meta)."""
    bar = "#------------------------------------------------------\n"
    date = date if date is not None else time.asctime()
    hx, hy, hz = (float(c) * float(field_strength) for c in field_unit)
    mx, my, mz = (float(c) for c in magnetization)
    with open(path, "w") as f:
        f.write(bar + "# Atomistic spin configuration file for vampire v5+\n" + bar)
        f.write(f"# Date: {date}\n" + bar)
        f.write(f"Time: {_g(time_s)}\n")
        f.write(f"Field: {_g(hx)}\t{_g(hy)}\t{_g(hz)}\n")
        f.write(f"Temperature: {_g(temperature)}\n")
        f.write(f"Magnetisation: {_g(mx)}\t{_g(my)}\t{_g(mz)}\n")
        f.write(bar + "Number of spin files: 1\n" + f"{data_name}\n" + bar)


class SpinSnapshots:
    """Writes numbered snapshots of a Simulation's output atoms.

    `atoms` is the output list (output_atom_list); each write() gathers the
    spins on the device (one copy of 24 bytes per output atom) and writes
    spins-<counter>.data and .meta into `directory`, as the reference's
    config::internal::atoms does with sim::output_atoms_file_counter."""

    def __init__(self, sim, atoms: np.ndarray, directory=".", binary: bool = True):
        self.sim = sim
        self.directory = Path(directory)
        self.binary = binary
        self.counter = 0
        sim.snapshot_setup(atoms)
        self._buf = np.empty(3 * int(np.asarray(atoms).size))

    def write(self, time_s: float, temperature: float, field_unit: Sequence[float], field_strength: float,
              magnetization: Sequence[float]) -> Path:
        data = self.sim.snapshot(out=self._buf)
        name = f"spins-{self.counter:08d}.data"
        path = self.directory / name
        (write_spins_binary if self.binary else write_spins_text)(path, data)
        write_spins_meta(self.directory / f"spins-{self.counter:08d}.meta", name, time_s, temperature,
                         field_unit, field_strength, magnetization)
        self.counter += 1
        return path
