"""ctypes binding of libvgpu.so (include/vgpu.h).

This is the Python side of the C ABI; it is what tests, bench.py and the
PyTorch adjoint wrapper call.  It never falls back to a CPU path: if the
shared library is missing or no CUDA device is present, calls raise
:class:`VGPUError`.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Optional, Tuple

import numpy as np

from .system import MATERIAL_DTYPE, SpinSystem

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libvgpu.so"

OK, ERR_ARG, ERR_CUDA, ERR_OOM, ERR_TIMEOUT, ERR_NAN, ERR_STATE = 0, -1, -2, -3, -4, -5, -6
PREC_FP32, PREC_FP64 = 0, 1
NOISE_PHILOX, NOISE_REPLAY = 0, 1
OPT_STORE_INCREMENT, OPT_STAGED_RECORDS, OPT_STAGE_SLICES, OPT_STAGE_BUFFERS, OPT_DIPOLE_FFT = 1, 2, 3, 4, 5
OPT_STAGE_WAIT_TEST = 6
OPT_COMPACT_RECORDS = 7
OPT_WINDOW_STAGING = 8
OPT_PROFILE_EVERY = 9
OPT_STAGE_WARPS = 10
EXCHANGE_FORMATS = ("iso_tab", "iso_bond", "vec_tab", "vec_bond", "dmi_tab", "tensor_bond")
RECORDS_NONE, RECORDS_WIDE, RECORDS_COMPACT, RECORDS_WINDOW = 0, 1, 2, 3
PASS_PREDICTOR, PASS_CORRECTOR = 0, 1
STATE_SPIN, STATE_PREDICTOR = 0, 1
DIPOLE_FAR_DIRECT, DIPOLE_FAR_FFT = 0, 1

_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)


class VGPUError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"vgpu error {code}: {msg}")
        self.code = code


class SystemDesc(C.Structure):
    _fields_ = [
        ("num_atoms", C.c_int32), ("num_materials", C.c_int32), ("exchange_type", C.c_int32),
        ("uniaxial_enabled", C.c_int32), ("cubic_enabled", C.c_int32), ("pad_", C.c_int32),
        ("num_bonds", C.c_int64), ("nl_start", _I32), ("nl_end", _I32), ("nl", _I32),
        ("nl_type", _I32), ("num_exchange", C.c_int64), ("jlist", _D), ("type", _I32),
        ("materials", C.c_void_p), ("sx", _D), ("sy", _D), ("sz", _D),
    ]


class SimParamsC(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("temperature", C.c_double), ("H_applied", C.c_double),
        ("H_vec", C.c_double * 3), ("thermal_enabled", C.c_int32), ("applied_enabled", C.c_int32),
        ("local_temperature", C.c_int32), ("local_applied_field", C.c_int32),
    ]


class AnisoExtC(C.Structure):
    _fields_ = [
        ("uniaxial_fourth", C.c_int32), ("uniaxial_sixth", C.c_int32), ("cubic_sixth", C.c_int32),
        ("cubic_rotation", C.c_int32), ("neel", C.c_int32), ("pad_", C.c_int32),
        ("ku4", _D), ("ku6", _D), ("kc6", _D), ("kc_basis", _D), ("neel_tensor", _D),
    ]


def _aniso_ext(a: dict):
    """AnisoExtC of SpinSystem.aniso; returns (struct, keep-alive list)."""
    keep = []

    def arr(v):
        if v is None:
            return C.cast(None, _D)
        v = np.ascontiguousarray(v, dtype=np.float64)
        keep.append(v)
        return _ptr(v, _D)

    x = AnisoExtC()
    x.uniaxial_fourth, x.uniaxial_sixth = int(a["u4"]), int(a["u6"])
    x.cubic_sixth, x.cubic_rotation, x.neel = int(a["c6"]), int(a["crot"]), int(a["neel"])
    x.ku4 = arr(a["ku4"] if a["u4"] else None)
    x.ku6 = arr(a["ku6"] if a["u6"] else None)
    x.kc6 = arr(a["kc6"] if a["c6"] else None)
    x.kc_basis = arr(a["kcb"] if a["crot"] else None)
    x.neel_tensor = arr(a["neel_tensor"] if a["neel"] else None)
    return x, keep


class BiquadDesc(C.Structure):
    _fields_ = [
        ("num_bonds", C.c_int64), ("nl_start", _I32), ("nl_end", _I32), ("nl", _I32), ("nl_type", _I32),
        ("num_exchange", C.c_int64), ("jlist", _D),
    ]


class DipoleDesc(C.Structure):
    _fields_ = [
        ("num_cells", C.c_int32), ("solver", C.c_int32), ("update_rate", C.c_int32), ("pad_", C.c_int32),
        ("macro_cell_size", C.c_double), ("cutoff", C.c_double), ("atom_cell", _I32), ("cell_pos_mom", _D),
        ("cell_volume", _D), ("cell_natoms", _I32), ("atom_x", _D), ("atom_y", _D), ("atom_z", _D),
    ]


_lib = None


def lib() -> C.CDLL:
    """Load libvgpu.so (built in-tree by vampire_b200.build)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise VGPUError(ERR_STATE, f"{LIB_PATH} not built; run python -m vampire_b200.build")
        _lib = C.CDLL(str(LIB_PATH))
        _lib.vgpu_version.restype = C.c_char_p
        _lib.vgpu_create.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        for name in ("vgpu_destroy",):
            getattr(_lib, name).argtypes = [C.c_void_p]
    return _lib


def version() -> str:
    return lib().vgpu_version().decode()


def _last_error(h) -> str:
    buf = C.create_string_buffer(1024)
    lib().vgpu_last_error(h, buf, C.c_size_t(len(buf)))
    return buf.value.decode(errors="replace")


def check(rc: int, h=None) -> None:
    if rc != OK:
        raise VGPUError(rc, _last_error(h))


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else C.cast(None, t)


def params_struct(p) -> SimParamsC:
    c = SimParamsC()
    c.dt = p.dt
    c.temperature = p.temperature
    c.H_applied = p.H_applied
    for k in range(3):
        c.H_vec[k] = float(p.H_vec[k])
    c.thermal_enabled = int(p.thermal)
    c.applied_enabled = int(p.applied)
    c.local_temperature = int(p.local_temperature)
    c.local_applied_field = int(p.local_applied_field)
    return c


def _desc(s: SpinSystem):
    """Fill a SystemDesc from a SpinSystem; returns (desc, keep-alive dict)."""
    keep = {}

    def arr(name, a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep[name] = a
        return a

    d = SystemDesc()
    d.num_atoms = s.n
    d.num_materials = s.num_materials
    d.exchange_type = s.exch_type
    d.uniaxial_enabled = int(s.uniaxial)
    d.cubic_enabled = int(s.cubic)
    d.num_bonds = s.num_bonds
    d.nl_start = _ptr(arr("st", s.nl_start, np.int32), _I32)
    d.nl_end = _ptr(arr("en", s.nl_end, np.int32), _I32)
    d.nl = _ptr(arr("nl", s.nl, np.int32), _I32)
    if s.nl_type is not None:
        d.nl_type = _ptr(arr("nt", s.nl_type, np.int32), _I32)
        w = {0: 1, 1: 3, 2: 9}[s.exch_type]
        d.num_exchange = s.jlist.size // w
    else:
        d.nl_type = C.cast(None, _I32)
        d.num_exchange = s.num_bonds
    d.jlist = _ptr(arr("jl", s.jlist, np.float64), _D)
    d.type = _ptr(arr("ty", s.type, np.int32), _I32)
    mats = arr("mats", s.materials, MATERIAL_DTYPE)
    d.materials = mats.ctypes.data
    sp = arr("sp", s.spins, np.float64)
    d.sx = _ptr(sp[0], _D)
    d.sy = _ptr(sp[1], _D)
    d.sz = _ptr(sp[2], _D)
    return d, keep


def validate_system(s: SpinSystem) -> None:
    """Host-only descriptor check (vgpu_validate_system); raises VGPUError."""
    d, keep = _desc(s)
    check(lib().vgpu_validate_system(C.byref(d)))


class Simulation:
    """One spin system resident on one GPU, driven through the C ABI."""

    def __init__(self, system: SpinSystem, device: int = 0, precision: str = "fp32",
                 noise_seed: int = 0):
        self.system = system
        self.n = system.n
        self.device = device
        self._h = C.c_void_p()
        prec = PREC_FP64 if precision == "fp64" else PREC_FP32
        check(lib().vgpu_create(device, prec, C.byref(self._h)))
        self.upload(system)
        self.set_params(system.params)
        self.set_noise(NOISE_PHILOX, noise_seed)

    # -- plumbing ----------------------------------------------------------
    @property
    def handle(self):
        return self._h

    def _check(self, rc):
        check(rc, self._h)

    def close(self) -> None:
        if self._h:
            lib().vgpu_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- system ------------------------------------------------------------
    def upload(self, s: SpinSystem) -> None:
        d, keep = _desc(s)
        self._check(lib().vgpu_upload_system(self._h, C.byref(d)))
        if s.aniso is not None:
            x, keep2 = _aniso_ext(s.aniso)
            self._check(lib().vgpu_set_anisotropy_ext(self._h, C.byref(x)))
        if s.biquadratic is not None:
            b = s.biquadratic
            keep3 = [np.ascontiguousarray(b[k], dtype=np.int32) for k in ("start", "end", "nl")]
            jl = np.ascontiguousarray(b["jlist"], dtype=np.float64)
            tp = None if b.get("type") is None else np.ascontiguousarray(b["type"], dtype=np.int32)
            q = BiquadDesc()
            q.num_bonds = keep3[2].size
            q.nl_start, q.nl_end, q.nl = (_ptr(keep3[0], _I32), _ptr(keep3[1], _I32), _ptr(keep3[2], _I32))
            q.nl_type = _ptr(tp, _I32) if tp is not None else C.cast(None, _I32)
            q.num_exchange = jl.size
            q.jlist = _ptr(jl, _D)
            self._check(lib().vgpu_set_biquadratic(self._h, C.byref(q)))

    def set_option(self, option: int, value: int) -> None:
        """vgpu_set_option: OPT_STORE_INCREMENT, OPT_STAGED_RECORDS, OPT_STAGE_SLICES,
        OPT_STAGE_BUFFERS, OPT_DIPOLE_FFT, OPT_STAGE_WAIT_TEST, OPT_COMPACT_RECORDS,
        OPT_WINDOW_STAGING, OPT_PROFILE_EVERY."""
        self._check(lib().vgpu_set_option(self._h, int(option), int(value)))

    def record_layout(self) -> Tuple[int, int]:
        """(RECORDS_NONE | RECORDS_WIDE | RECORDS_COMPACT | RECORDS_WINDOW, coupling
        dictionary entries)."""
        lay, nd = C.c_int32(), C.c_int32()
        self._check(lib().vgpu_record_layout(self._h, C.byref(lay), C.byref(nd)))
        return lay.value, nd.value

    def exchange_format(self) -> str:
        """Per-bond exchange format chosen at upload: iso_tab, iso_bond,
        vec_tab, vec_bond, dmi_tab or tensor_bond."""
        f = C.c_int32()
        self._check(lib().vgpu_exchange_format(self._h, C.byref(f)))
        return EXCHANGE_FORMATS[f.value]

    def set_params(self, p) -> None:
        c = params_struct(p)
        self._check(lib().vgpu_set_params(self._h, C.byref(c)))

    # -- spins -------------------------------------------------------------
    def spins(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Current spins as (3, n) float64; `out` (e.g. a view of pinned host
        memory) is filled in place when given."""
        if out is None:
            out = np.empty((3, self.n))
        assert out.shape == (3, self.n) and out.dtype == np.float64 and out[0].flags.c_contiguous
        self._check(lib().vgpu_get_spins(self._h, _ptr(out[0], _D), _ptr(out[1], _D), _ptr(out[2], _D)))
        return out

    def set_spins(self, s: np.ndarray) -> None:
        s = np.ascontiguousarray(s, dtype=np.float64)
        self._check(lib().vgpu_set_spins(self._h, _ptr(s[0], _D), _ptr(s[1], _D), _ptr(s[2], _D)))

    def fields(self) -> np.ndarray:
        out = np.empty((3, self.n))
        self._check(lib().vgpu_get_fields(self._h, _ptr(out[0], _D), _ptr(out[1], _D), _ptr(out[2], _D)))
        return out

    # -- integration -------------------------------------------------------
    def set_noise(self, mode: int, seed: int = 0) -> None:
        self._check(lib().vgpu_set_noise(self._h, C.c_int(mode), C.c_uint64(seed)))

    def set_noise_replay(self, xi: np.ndarray) -> None:
        xi = np.ascontiguousarray(xi, dtype=np.float64)
        assert xi.size == 3 * self.n
        self._check(lib().vgpu_set_noise_replay(self._h, _ptr(xi, _D)))

    def thermal_noise(self, step: int) -> np.ndarray:
        """The 3n Philox Gaussians the kernels use at `step` (x|y|z blocks)."""
        out = np.empty(3 * self.n)
        self._check(lib().vgpu_thermal_noise(self._h, C.c_uint64(step), _ptr(out, _D)))
        return out

    @property
    def step(self) -> int:
        v = C.c_uint64()
        self._check(lib().vgpu_get_step(self._h, C.byref(v)))
        return v.value

    @step.setter
    def step(self, v: int) -> None:
        self._check(lib().vgpu_set_step(self._h, C.c_uint64(v)))

    def llg_heun(self, n_steps: int = 1) -> None:
        self._check(lib().vgpu_llg_heun(self._h, C.c_uint64(n_steps)))

    def llg_midpoint(self, n_steps: int = 1) -> None:
        """n_steps of the LLG-Midpoint integrator (vgpu_llg_midpoint)."""
        self._check(lib().vgpu_llg_midpoint(self._h, C.c_uint64(n_steps)))

    # -- shards ------------------------------------------------------------
    def llg_pass(self, which: int) -> None:
        """One fused pass: PASS_PREDICTOR or PASS_CORRECTOR (vgpu_llg_pass)."""
        self._check(lib().vgpu_llg_pass(self._h, C.c_int(which)))

    def llg_pass_range(self, which: int, first: int, end: int) -> None:
        """One pass over the updated atoms first..end-1 (first a multiple of
        32; vgpu_llg_pass_range)."""
        self._check(lib().vgpu_llg_pass_range(self._h, C.c_int(which), C.c_int32(first), C.c_int32(end)))

    def set_owned(self, n_owned: int, noise_base: int = 0) -> None:
        self._check(lib().vgpu_set_owned(self._h, C.c_int32(n_owned), C.c_int64(noise_base)))

    def halo_pack(self, which: int, idx_ptr: int, count: int, out_ptr: int) -> None:
        """Device pointers: idx (int32[count]) -> out (3*count values)."""
        self._check(lib().vgpu_halo_pack(self._h, C.c_int(which), C.c_void_p(idx_ptr), C.c_int32(count),
                                         C.c_void_p(out_ptr)))

    def halo_unpack(self, which: int, first: int, count: int, in_ptr: int) -> None:
        self._check(lib().vgpu_halo_unpack(self._h, C.c_int(which), C.c_int32(first), C.c_int32(count),
                                           C.c_void_p(in_ptr)))

    def halo_pack_on(self, which: int, idx_ptr: int, count: int, out_ptr: int, stream: int) -> None:
        """halo_pack on another stream (a cudaStream_t as an integer)."""
        self._check(lib().vgpu_halo_pack_on(self._h, C.c_int(which), C.c_void_p(idx_ptr), C.c_int32(count),
                                            C.c_void_p(out_ptr), C.c_void_p(stream)))

    def halo_unpack_on(self, which: int, first: int, count: int, in_ptr: int, stream: int) -> None:
        self._check(lib().vgpu_halo_unpack_on(self._h, C.c_int(which), C.c_int32(first), C.c_int32(count),
                                              C.c_void_p(in_ptr), C.c_void_p(stream)))

    def stats_copy_rows(self, mask_id: int, out_ptr: int) -> None:
        """Enqueue a copy of the latest rows (9 doubles per bin) to out_ptr
        (pinned host or device memory) on the library stream; no wait."""
        self._check(lib().vgpu_stats_copy_rows(self._h, C.c_int32(mask_id), C.c_void_p(out_ptr)))

    def snapshot_setup(self, atoms) -> None:
        """Output atom list of the spin snapshots (vgpu_snapshot_setup)."""
        a = np.ascontiguousarray(atoms, dtype=np.int64)
        self._snap_n = int(a.size)
        self._check(lib().vgpu_snapshot_setup(self._h, a.ctypes.data_as(C.POINTER(C.c_int64)),
                                              C.c_int64(a.size)))

    def snapshot(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """The listed atoms' spins, x y z interleaved in FP64 (the data block
        of the binary spin file), gathered on the device (vgpu_snapshot).
        `out` (e.g. a view of pinned host memory) is filled in place."""
        n = getattr(self, "_snap_n", None)
        if n is None:
            raise VGPUError(ERR_STATE, "snapshot_setup not called")
        if out is None:
            out = np.empty(3 * n)
        assert out.dtype == np.float64 and out.size == 3 * n and out.flags.c_contiguous
        self._check(lib().vgpu_snapshot(self._h, _ptr(out, _D)))
        self.synchronize()
        return out

    def stats_derived(self, mask_id: int, temperature: float):
        """(susceptibility (size, 4), specific heat (size,), std dev (size, 4))
        of the updates since the last reset (vgpu_stats_get_derived)."""
        size = self._mask_sizes[mask_id]
        sus, sh, sd = np.zeros(4 * size), np.zeros(size), np.zeros(4 * size)
        self._check(lib().vgpu_stats_get_derived(self._h, C.c_int32(mask_id), C.c_double(temperature),
                                                 _ptr(sus, _D), _ptr(sh, _D), _ptr(sd, _D)))
        return sus.reshape(size, 4), sh, sd.reshape(size, 4)

    def torque_update(self) -> None:
        """System and per-material torque of the current state, added to the
        running means (vgpu_torque_update)."""
        self._check(lib().vgpu_torque_update(self._h))

    def torque(self) -> dict:
        """{total[3], mean[3], material[M,3], material_mean[M,3], max, count}."""
        M = self.system.materials.size
        tot, mean = np.zeros(3), np.zeros(3)
        mat, mmean = np.zeros(3 * M), np.zeros(3 * M)
        mx, cnt = C.c_double(), C.c_int64()
        self._check(lib().vgpu_torque_get(self._h, _ptr(tot, _D), _ptr(mean, _D), _ptr(mat, _D), _ptr(mmean, _D),
                                          C.byref(mx), C.byref(cnt)))
        return {"total": tot, "mean": mean, "material": mat.reshape(M, 3), "material_mean": mmean.reshape(M, 3),
                "max": mx.value, "count": cnt.value}

    def torque_reset(self) -> None:
        self._check(lib().vgpu_torque_reset(self._h))

    def stats_sums(self, mask_id: int, size: int) -> np.ndarray:
        """Raw per-bin sums of the last statistics update, (size, 8)."""
        out = np.zeros((size, 8))
        self._check(lib().vgpu_stats_get_sums(self._h, C.c_int32(mask_id), _ptr(out, _D)))
        return out

    # -- dipole field --------------------------------------------------------
    @staticmethod
    def _dipole_desc(cells: dict, keep: dict) -> "DipoleDesc":

        def arr(name, a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep[name] = a
            return a

        d = DipoleDesc()
        d.num_cells = int(np.asarray(cells["cell_natoms"]).size)
        d.solver = 1 if cells.get("solver", "tensor") == "tensor" else 0
        d.update_rate = int(cells.get("update_rate", 100))
        d.macro_cell_size = float(cells["macro_cell_size"])
        d.cutoff = float(cells.get("cutoff", 2.0))
        d.atom_cell = _ptr(arr("ac", cells["atom_cell"], np.int32), _I32)
        d.cell_pos_mom = _ptr(arr("cp", cells["cell_pos_mom"], np.float64), _D)
        d.cell_volume = _ptr(arr("cv", cells["cell_volume"], np.float64), _D)
        d.cell_natoms = _ptr(arr("cn", cells["cell_natoms"], np.int32), _I32)
        if "coords" in cells and cells["coords"] is not None:
            c = arr("xyz", cells["coords"], np.float64)
            d.atom_x, d.atom_y, d.atom_z = _ptr(c[0], _D), _ptr(c[1], _D), _ptr(c[2], _D)
        return d

    def dipole_setup(self, cells: dict) -> None:
        """cells: atom_cell, cell_pos_mom, cell_volume, cell_natoms,
        macro_cell_size, cutoff, update_rate, solver ('tensor'|'macrocell'),
        coords (3, n) for the tensor solver (the reference's cells:: data)."""
        keep = {}
        d = self._dipole_desc(cells, keep)
        self._ncells = d.num_cells
        self._check(lib().vgpu_dipole_setup(self._h, C.byref(d)))

    def dipole_setup_shard(self, whole_cells: dict, global_type: np.ndarray, local_ids: np.ndarray) -> None:
        """The dipole solver on a shard (vgpu_dipole_setup_shard): whole_cells
        are the whole system's cells (dipole_setup's keys; atom_cell and
        coords of every global atom), global_type the material id of every
        global atom, local_ids the global id of each of the shard's atoms.
        The field then waits for the moment sum over ranks (dipole_finish)."""
        keep = {}
        d = self._dipole_desc(whole_cells, keep)
        gt = np.ascontiguousarray(global_type, dtype=np.int32)
        loc = np.ascontiguousarray(local_ids, dtype=np.int64)
        self._ncells = d.num_cells
        self._check(lib().vgpu_dipole_setup_shard(self._h, C.byref(d), C.c_int64(gt.size), _ptr(gt, _I32),
                                                  loc.ctypes.data_as(C.POINTER(C.c_int64))))

    def dipole_moment_buffer(self) -> Tuple[int, int]:
        """(device pointer, count) of the FP64 cell moment buffer (x|y|z blocks)."""
        p, n = C.POINTER(C.c_double)(), C.c_int64()
        self._check(lib().vgpu_dipole_moment_buffer(self._h, C.byref(p), C.byref(n)))
        return C.cast(p, C.c_void_p).value or 0, n.value

    def dipole_moment_tensor(self):
        """The cell moment buffer as a torch CUDA tensor (no copy), for an
        in-place all-reduce over ranks."""
        import torch
        ptr, count = self.dipole_moment_buffer()

        class _Buf:
            __cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False),
                                        "version": 3, "strides": None}

        return torch.as_tensor(_Buf(), device=torch.device("cuda", self.device))

    def dipole_pending(self) -> bool:
        p = C.c_int32()
        self._check(lib().vgpu_dipole_pending(self._h, C.byref(p)))
        return bool(p.value)

    def dipole_finish(self) -> None:
        self._check(lib().vgpu_dipole_finish(self._h))

    def dipole_update(self) -> None:
        self._check(lib().vgpu_dipole_update(self._h))

    def dipole_method(self) -> int:
        """DIPOLE_FAR_DIRECT or DIPOLE_FAR_FFT (far-field method chosen at setup)."""
        m = C.c_int32()
        self._check(lib().vgpu_dipole_method(self._h, C.byref(m)))
        return m.value

    def dipole_cells(self):
        """(moments J/T, B field T, mu0 Hd field T), each (3, ncells)."""
        nc = self._ncells
        m, b, hd = np.empty(3 * nc), np.empty(3 * nc), np.empty(3 * nc)
        self._check(lib().vgpu_dipole_get_cells(self._h, _ptr(m, _D), _ptr(b, _D), _ptr(hd, _D)))
        return m.reshape(3, nc), b.reshape(3, nc), hd.reshape(3, nc)

    def set_dipole_field(self, b: np.ndarray, hd: Optional[np.ndarray] = None) -> None:
        b = np.ascontiguousarray(b, dtype=np.float64)
        h = np.ascontiguousarray(hd, dtype=np.float64) if hd is not None else None
        self._check(lib().vgpu_set_dipole_field(self._h, _ptr(b[0], _D), _ptr(b[1], _D), _ptr(b[2], _D),
                                                _ptr(h[0] if h is not None else None, _D),
                                                _ptr(h[1] if h is not None else None, _D),
                                                _ptr(h[2] if h is not None else None, _D)))

    # -- Monte Carlo -------------------------------------------------------
    def mc_setup(self, colour: Optional[np.ndarray] = None) -> int:
        nc = C.c_int32()
        c = np.ascontiguousarray(colour, dtype=np.int32) if colour is not None else None
        self._check(lib().vgpu_mc_setup(self._h, _ptr(c, _I32), C.byref(nc)))
        return nc.value

    def mc_colours(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.int32)
        self._check(lib().vgpu_mc_get_colours(self._h, _ptr(out, _I32)))
        return out

    def mc_set_replay(self, rnd: Optional[np.ndarray]) -> None:
        r = np.ascontiguousarray(rnd, dtype=np.float64) if rnd is not None else None
        self._check(lib().vgpu_mc_set_replay(self._h, _ptr(r, _D)))

    def mc_sweep(self, n_sweeps: int = 1) -> None:
        self._check(lib().vgpu_mc_sweep(self._h, C.c_uint64(n_sweeps)))

    def mc_colour(self, colour: int) -> None:
        """One colour of the current sweep (vgpu_mc_colour; colours in order)."""
        self._check(lib().vgpu_mc_colour(self._h, C.c_int32(colour)))

    def mc_set_sweep(self, sweep: int) -> None:
        self._check(lib().vgpu_mc_set_sweep(self._h, C.c_uint64(sweep)))

    def mc_counters(self):
        mv, rj = C.c_double(), C.c_double()
        self._check(lib().vgpu_mc_counters(self._h, C.byref(mv), C.byref(rj)))
        return mv.value, rj.value

    # -- statistics --------------------------------------------------------
    # -- constrained Monte Carlo ------------------------------------------
    def cmc_setup(self, phi_deg: float, theta_deg: float, init_spins: bool = True) -> None:
        """Constraint direction (phi from z, theta about z, degrees) and, with
        init_spins, every spin along it (the reference's CMCinit)."""
        self._check(lib().vgpu_cmc_setup(self._h, C.c_double(phi_deg), C.c_double(theta_deg),
                                          C.c_int32(int(init_spins))))

    def cmc_setup_materials(self, constrained, phi_deg, theta_deg, init_spins: bool = True) -> None:
        """Hybrid constrained Monte Carlo: per material a constraint flag and
        direction (degrees); constrained materials' spins along it with
        init_spins (the reference's CMCMCinit)."""
        M = self.system.materials.size
        c = np.ascontiguousarray(constrained, dtype=np.int32).reshape(M)
        ph = np.ascontiguousarray(phi_deg, dtype=np.float64).reshape(M)
        th = np.ascontiguousarray(theta_deg, dtype=np.float64).reshape(M)
        self._check(lib().vgpu_cmc_setup_materials(self._h, _ptr(c, _I32), _ptr(ph, _D), _ptr(th, _D),
                                                   C.c_int32(int(init_spins))))

    def cmc_material_moments(self) -> np.ndarray:
        """Running moments [M, 3] (mu_B) of the constrained materials (hybrid)."""
        M = self.system.materials.size
        out = np.zeros(3 * M)
        self._check(lib().vgpu_cmc_material_moments(self._h, _ptr(out, _D)))
        return out.reshape(M, 3)

    def cmc_sweep(self, n_steps: int = 1) -> None:
        """n_steps constrained Monte Carlo steps (about N pair moves each)."""
        self._check(lib().vgpu_cmc_sweep(self._h, C.c_uint64(n_steps)))

    def cmc_pairs(self, pairs: np.ndarray, rnd: np.ndarray, moment: Optional[np.ndarray] = None) -> None:
        """One phase on explicit pairs (all atoms of one colour, each once) with
        given random numbers rnd[4K] (Gaussians x|y|z of K, then uniforms)."""
        pr = np.ascontiguousarray(pairs, dtype=np.int32).ravel()
        r = np.ascontiguousarray(rnd, dtype=np.float64)
        mm = None if moment is None else np.ascontiguousarray(moment, dtype=np.float64)
        self._check(lib().vgpu_cmc_pairs(self._h, _ptr(pr, _I32), C.c_int32(pr.size // 2), _ptr(r, _D),
                                         _ptr(mm, _D) if mm is not None else C.cast(None, _D)))

    def cmc_state(self):
        """(total moment [3] in mu_B, [pair moves, accepted, energy rejections,
        sphere rejections])."""
        m, c = np.zeros(3), np.zeros(4)
        self._check(lib().vgpu_cmc_get(self._h, _ptr(m, _D), _ptr(c, _D)))
        return m, c

    def cmc_frame(self):
        """(P[3,3] rotating the constraint direction to z, constraint vector)."""
        P, v = np.zeros(9), np.zeros(3)
        self._check(lib().vgpu_cmc_frame(self._h, _ptr(P, _D), _ptr(v, _D)))
        return P.reshape(3, 3), v

    def add_mask(self, mask: np.ndarray, size: int) -> int:
        m = np.ascontiguousarray(mask, dtype=np.int32)
        out = C.c_int32()
        self._check(lib().vgpu_stats_add_mask(self._h, _ptr(m, _I32), C.c_int32(size), C.byref(out)))
        self._mask_sizes = getattr(self, "_mask_sizes", {})
        self._mask_sizes[out.value] = size
        return out.value

    def stats_update(self, magnetization: bool = True, energy: bool = False) -> None:
        self._check(lib().vgpu_stats_update(self._h, C.c_int32(int(magnetization) | (int(energy) << 1))))

    def magnetization(self, mask_id: int = 0):
        size = self._mask_sizes[mask_id]
        m = np.empty(4 * size)
        mean = np.empty(4 * size)
        cnt = C.c_int64()
        self._check(lib().vgpu_stats_get_magnetization(self._h, C.c_int32(mask_id), _ptr(m, _D), _ptr(mean, _D),
                                                       C.byref(cnt)))
        return m, mean, cnt.value

    def energy(self, mask_id: int = 0):
        size = self._mask_sizes[mask_id]
        e = np.empty(5 * size)
        mean = np.empty(5 * size)
        cnt = C.c_int64()
        self._check(lib().vgpu_stats_get_energy(self._h, C.c_int32(mask_id), _ptr(e, _D), _ptr(mean, _D),
                                                C.byref(cnt)))
        return e, mean, cnt.value

    def stats_reset(self) -> None:
        self._check(lib().vgpu_stats_reset(self._h))

    # -- streams and timing -----------------------------------------------
    def stream_ptr(self) -> int:
        p = C.c_void_p()
        self._check(lib().vgpu_get_stream(self._h, C.byref(p)))
        return p.value or 0

    def synchronize(self) -> None:
        self._check(lib().vgpu_synchronize(self._h))

    def profile(self, enable: bool) -> None:
        self._check(lib().vgpu_profile(self._h, C.c_int(int(enable))))

    PROF_KINDS = ("predictor", "corrector", "statistics", "dipole", "monte_carlo", "other")

    def profile_read(self) -> dict:
        ms = np.zeros(6)
        cnt = np.zeros(6, dtype=np.int64)
        launches = C.c_int64()
        self._check(lib().vgpu_profile_read(self._h, _ptr(ms, _D), cnt.ctypes.data_as(C.POINTER(C.c_int64)),
                                            C.c_int32(6), C.byref(launches)))
        out = {k: {"ms": float(ms[i]), "count": int(cnt[i])} for i, k in enumerate(self.PROF_KINDS)}
        out["kernel_launches"] = launches.value
        return out
