"""Oracle access for tests, smoke() and the CPU baseline of bench.py.

TEST INFRASTRUCTURE ONLY.  Two checkers live here:

* ``liboracle.so`` -- oracle/vref.c, the FP64 CPU restatement of the
  reference spin update (compiled with gcc on first use, or by
  ``__graft_entry__.build()``);
* ``vampire-harness`` -- the reference program's own objects driven by
  oracle/harness.cpp (built by oracle/build_ref.py where the reference tree
  is present).  Fixtures it produced are committed under tests/golden/.

The product (vampire_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
LIB_PATH = HERE / "liboracle.so"
HARNESS = HERE / "_ref" / "vampire-harness"
SERIAL = HERE / "_ref" / "vampire-serial"

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


class VRefSys(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("nmat", C.c_int), ("exch_type", C.c_int),
        ("uniaxial", C.c_int), ("cubic", C.c_int), ("thermal", C.c_int), ("applied", C.c_int),
        ("pad_", C.c_int),
        ("start", _I), ("end", _I), ("nl", _I), ("nltype", _I), ("jlist", _D), ("type", _I),
        ("A", _D), ("B", _D), ("sigma", _D), ("ku2", _D), ("kux", _D), ("kuy", _D), ("kuz", _D),
        ("kc4", _D), ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double), ("hloc", _D),
        ("hdx", _D), ("hdy", _D), ("hdz", _D), ("hmx", _D), ("hmy", _D), ("hmz", _D),
        ("dt", C.c_double), ("half_dt", C.c_double), ("H_applied", C.c_double),
        ("H_vec", C.c_double * 3), ("mus", _D), ("mus_SI", _D),
        ("u4", C.c_int), ("u6", C.c_int), ("c6", C.c_int), ("crot", C.c_int), ("neel", C.c_int),
        ("pad2_", C.c_int), ("ku4", _D), ("ku6", _D), ("kc6", _D), ("kcb", _D), ("neelt", _D),
        ("bq_start", _I), ("bq_end", _I), ("bq_nl", _I), ("bq_type", _I), ("bq_j", _D),
    ]


def build_lib(force: bool = False) -> Path:
    src = HERE / "vref.c"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        cmd = ["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(LIB_PATH), str(src), "-lm"]
        subprocess.run(cmd, check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build_lib()
        _lib = C.CDLL(str(LIB_PATH))
        for name in ("vref_spin_fields", "vref_external_fields", "vref_llg_heun", "vref_magnetization",
                     "vref_heun_predict", "vref_heun_correct",
                     "vref_energy", "vref_spin_energy"):
            getattr(_lib, name).restype = None
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else C.cast(None, t)


class OracleSystem:
    """A vref_sys view of a vampire_b200.system.SpinSystem (arrays kept alive)."""

    def __init__(self, s, dipole_field=None, demag_field=None):
        self.s = s
        m = s.materials
        p = s.params
        keep = {}

        def arr(name, a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep[name] = a
            return a

        st = VRefSys()
        st.n = s.n
        st.nmat = m.size
        st.exch_type = s.exch_type
        st.uniaxial = int(s.uniaxial)
        st.cubic = int(s.cubic)
        st.thermal = int(p.thermal)
        st.applied = int(p.applied)
        st.start = _p(arr("start", s.nl_start, np.int32), _I)
        st.end = _p(arr("end", s.nl_end, np.int32), _I)
        st.nl = _p(arr("nl", s.nl, np.int32), _I)
        st.nltype = _p(arr("nltype", s.nl_type, np.int32), _I) if s.nl_type is not None else _p(None, _I)
        st.jlist = _p(arr("jlist", s.jlist, np.float64), _D)
        st.type = _p(arr("type", s.type, np.int32), _I)
        st.A = _p(arr("A", m["one_oneplusalpha_sq"], np.float64), _D)
        st.B = _p(arr("B", m["alpha_oneplusalpha_sq"], np.float64), _D)
        st.sigma = _p(arr("sigma", s.sigma(), np.float64), _D)
        st.ku2 = _p(arr("ku2", m["ku2"], np.float64), _D)
        kv = arr("kv", m["ku_vector"], np.float64)
        st.kux = _p(arr("kux", kv[:, 0], np.float64), _D)
        st.kuy = _p(arr("kuy", kv[:, 1], np.float64), _D)
        st.kuz = _p(arr("kuz", kv[:, 2], np.float64), _D)
        st.kc4 = _p(arr("kc4", m["kc4"], np.float64), _D)
        hv = np.asarray(p.H_vec, dtype=np.float64)
        st.hx, st.hy, st.hz = (p.H_vec[0] * p.H_applied, p.H_vec[1] * p.H_applied, p.H_vec[2] * p.H_applied)
        st.hloc = _p(arr("hloc", m["applied_field"], np.float64), _D) if p.local_applied_field else _p(None, _D)
        if dipole_field is not None:
            st.hdx = _p(arr("hdx", dipole_field[0], np.float64), _D)
            st.hdy = _p(arr("hdy", dipole_field[1], np.float64), _D)
            st.hdz = _p(arr("hdz", dipole_field[2], np.float64), _D)
        if demag_field is not None:
            st.hmx = _p(arr("hmx", demag_field[0], np.float64), _D)
            st.hmy = _p(arr("hmy", demag_field[1], np.float64), _D)
            st.hmz = _p(arr("hmz", demag_field[2], np.float64), _D)
        st.dt = p.dt
        st.half_dt = 0.5 * p.dt
        st.H_applied = p.H_applied
        for k in range(3):
            st.H_vec[k] = hv[k]
        st.mus = _p(arr("mus", m["mu_s_SI"] / 9.27400915e-24, np.float64), _D)
        st.mus_SI = _p(arr("mus_SI", m["mu_s_SI"], np.float64), _D)
        bq = getattr(s, "biquadratic", None)
        if bq is not None:
            st.bq_start = _p(arr("bq_start", bq["start"], np.int32), _I)
            st.bq_end = _p(arr("bq_end", bq["end"], np.int32), _I)
            st.bq_nl = _p(arr("bq_nl", bq["nl"], np.int32), _I)
            if bq.get("type") is not None:
                st.bq_type = _p(arr("bq_type", bq["type"], np.int32), _I)
            st.bq_j = _p(arr("bq_j", bq["jlist"], np.float64), _D)
        a = getattr(s, "aniso", None)
        if a is not None:
            st.u4, st.u6, st.c6, st.crot, st.neel = (int(a["u4"]), int(a["u6"]), int(a["c6"]), int(a["crot"]),
                                                     int(a["neel"]))
            for key, f in (("ku4", "ku4"), ("ku6", "ku6"), ("kc6", "kc6"), ("kcb", "kcb"), ("neel_tensor", "neelt")):
                if a.get(key) is not None:
                    setattr(st, f, _p(arr(key, a[key], np.float64), _D))
        self.st = st
        self.keep = keep

    # -- adjoint (FP64 CPU) ---------------------------------------------------
    def adjoint(self, spins, target, w, every=0):
        """(loss, grad[5]) of L = sum_t w (m_z(t) - target_t)^2 over
        len(target) steps; grad = dL/d(exchange scale), dL/dKu_SI, dL/dH (3)."""
        s = np.ascontiguousarray(spins, dtype=np.float64)
        tg = np.ascontiguousarray(target, dtype=np.float64)
        g = np.zeros(5)
        lib().vref_adjoint.restype = C.c_double
        loss = lib().vref_adjoint(C.byref(self.st), _p(s[0], _D), _p(s[1], _D), _p(s[2], _D),
                                  C.c_int64(tg.size), _p(tg, _D), C.c_double(w), C.c_int64(every), _p(g, _D))
        return loss, g

    def trajectory_loss(self, spins, target, w):
        s = np.ascontiguousarray(spins, dtype=np.float64)
        tg = np.ascontiguousarray(target, dtype=np.float64)
        lib().vref_trajectory_loss.restype = C.c_double
        return lib().vref_trajectory_loss(C.byref(self.st), _p(s[0], _D), _p(s[1], _D), _p(s[2], _D),
                                          C.c_int64(tg.size), _p(tg, _D), C.c_double(w))

    def mz_trajectory(self, spins, nsteps):
        s = np.ascontiguousarray(spins, dtype=np.float64)
        out = np.zeros(nsteps)
        lib().vref_mz_trajectory(C.byref(self.st), _p(s[0], _D), _p(s[1], _D), _p(s[2], _D),
                                 C.c_int64(nsteps), _p(out, _D))
        return out

    def llg_heun(self, spins: np.ndarray, n_steps: int, xi: Optional[np.ndarray] = None) -> np.ndarray:
        s = np.ascontiguousarray(spins, dtype=np.float64).copy()
        xi_c = np.ascontiguousarray(xi, dtype=np.float64) if xi is not None else None
        lib().vref_llg_heun(C.byref(self.st), _p(s[0], _D), _p(s[1], _D), _p(s[2], _D),
                            _p(xi_c, _D), C.c_int64(n_steps))
        return s

    def llg_midpoint(self, spins: np.ndarray, n_steps: int, xi: Optional[np.ndarray] = None) -> np.ndarray:
        """n_steps of sim::LLG_Midpoint (vref_llg_midpoint)."""
        s = np.ascontiguousarray(spins, dtype=np.float64).copy()
        xi_c = np.ascontiguousarray(xi, dtype=np.float64) if xi is not None else None
        alpha = np.ascontiguousarray(self.s.materials["alpha"], dtype=np.float64)
        lib().vref_llg_midpoint.restype = None
        lib().vref_llg_midpoint(C.byref(self.st), _p(s[0], _D), _p(s[1], _D), _p(s[2], _D), _p(xi_c, _D),
                                _p(alpha, _D), C.c_int64(n_steps))
        return s

    def heun_predict(self, spins: np.ndarray, xi: Optional[np.ndarray] = None):
        """Predictor half of one step (vref_heun_predict): returns (s', keep),
        keep being the 12n state the corrector half needs."""
        s = np.ascontiguousarray(spins, dtype=np.float64)
        xi_c = np.ascontiguousarray(xi, dtype=np.float64) if xi is not None else None
        p = np.zeros((3, self.s.n))
        keep = np.zeros(12 * self.s.n)
        lib().vref_heun_predict(C.byref(self.st), _p(s[0], _D), _p(s[1], _D), _p(s[2], _D), _p(xi_c, _D),
                                _p(p[0], _D), _p(p[1], _D), _p(p[2], _D), _p(keep, _D))
        return p, keep

    def heun_correct(self, spins: np.ndarray, p: np.ndarray, keep: np.ndarray) -> np.ndarray:
        """Corrector half (vref_heun_correct): s1 from s0 = spins, s' = p."""
        s = np.ascontiguousarray(spins, dtype=np.float64).copy()
        pc = np.ascontiguousarray(p, dtype=np.float64)
        lib().vref_heun_correct(C.byref(self.st), _p(s[0], _D), _p(s[1], _D), _p(s[2], _D), _p(pc[0], _D),
                                _p(pc[1], _D), _p(pc[2], _D), _p(keep, _D))
        return s

    def spin_fields(self, spins: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(spins, dtype=np.float64)
        h = np.zeros((3, self.s.n))
        lib().vref_spin_fields(C.byref(self.st), _p(s[0], _D), _p(s[1], _D), _p(s[2], _D),
                               _p(h[0], _D), _p(h[1], _D), _p(h[2], _D))
        return h

    def external_fields(self, xi=None) -> np.ndarray:
        h = np.zeros((3, self.s.n))
        xi_c = np.ascontiguousarray(xi, dtype=np.float64) if xi is not None else None
        lib().vref_external_fields(C.byref(self.st), _p(xi_c, _D), _p(h[0], _D), _p(h[1], _D),
                                   _p(h[2], _D))
        return h

    def mc_params(self):
        """Per-material (sigma, kBTBohr, mu_s/muB) of the angle move
        (src/montecarlo/mc.cpp:45-53) at the system temperature."""
        p, m = self.s.params, self.s.materials
        sig, beta, ratio = [], [], []
        for k in range(m.size):
            T = m[k]["temperature"] if p.local_temperature else p.temperature
            a, Tc = m[k]["temperature_rescaling_alpha"], m[k]["temperature_rescaling_Tc"]
            Tr = Tc * (T / Tc) ** a if T < Tc else T
            b = 9.27400915e-24 / (Tr * 1.3806503e-23) if Tr > 0 else np.inf
            sig.append(0.02 if Tr < 1.0 else (1.0 / b) ** 0.2 * 0.08)
            beta.append(b)
            ratio.append(m[k]["mu_s_SI"] * 1.07828231e23)
        return np.array(sig), np.array(beta), np.array(ratio)

    def mc_colour_sweep(self, spins, colour, rnd):
        """One colour-ordered Metropolis sweep with given random numbers (4n)."""
        s = np.ascontiguousarray(spins, dtype=np.float64).copy()
        colour = np.asarray(colour)
        nc = int(colour.max()) + 1
        order = np.ascontiguousarray(np.argsort(colour, kind="stable"), dtype=np.int32)
        off = np.ascontiguousarray(np.r_[0, np.cumsum(np.bincount(colour, minlength=nc))], dtype=np.int32)
        sig, beta, ratio = self.mc_params()
        r = np.ascontiguousarray(rnd, dtype=np.float64)
        lib().vref_mc_colour_sweep.restype = C.c_long
        rej = lib().vref_mc_colour_sweep(C.byref(self.st), _p(s[0], _D), _p(s[1], _D), _p(s[2], _D),
                                         _p(order, _I), _p(off, _I), C.c_int(nc), _p(r, _D), _p(sig, _D),
                                         _p(beta, _D), _p(ratio, _D))
        return s, int(rej)

    def mc_pass(self, spins, atoms, rnd):
        """Metropolis moves of the listed atoms, in order, with given random
        numbers (4n: x|y|z Gaussians, acceptance uniforms); the pass of one
        colour of a sweep over one shard's owned atoms."""
        s = np.ascontiguousarray(spins, dtype=np.float64).copy()
        order = np.ascontiguousarray(atoms, dtype=np.int32)
        off = np.array([0, order.size], dtype=np.int32)
        sig, beta, ratio = self.mc_params()
        r = np.ascontiguousarray(rnd, dtype=np.float64)
        lib().vref_mc_colour_sweep.restype = C.c_long
        rej = lib().vref_mc_colour_sweep(C.byref(self.st), _p(s[0], _D), _p(s[1], _D), _p(s[2], _D),
                                         _p(order, _I), _p(off, _I), C.c_int(1), _p(r, _D), _p(sig, _D),
                                         _p(beta, _D), _p(ratio, _D))
        return s, int(rej)

    def cmc_pairs(self, spins, pairs, rnd, P, pv, M):
        """The reference's constrained pair-move rule (vref_cmc_pairs) on the
        given ordered pairs with given random numbers; returns (spins, M,
        [accepted, energy rejections, sphere rejections])."""
        s = np.ascontiguousarray(spins, dtype=np.float64).copy()
        pr = np.ascontiguousarray(pairs, dtype=np.int32).ravel()
        r = np.ascontiguousarray(rnd, dtype=np.float64)
        Pm = np.ascontiguousarray(P, dtype=np.float64).ravel()
        v = np.ascontiguousarray(pv, dtype=np.float64)
        m = np.ascontiguousarray(M, dtype=np.float64).copy()
        sig, beta, ratio = self.mc_params()
        cnt = np.zeros(3, dtype=np.int64)
        lib().vref_cmc_pairs.restype = None
        lib().vref_cmc_pairs(C.byref(self.st), _p(s[0], _D), _p(s[1], _D), _p(s[2], _D), _p(pr, _I),
                             C.c_int(pr.size // 2), _p(r, _D), _p(Pm, _D), _p(v, _D), _p(m, _D), _p(sig, _D),
                             _p(beta, _D), _p(ratio, _D), cnt.ctypes.data_as(C.POINTER(C.c_long)))
        return s, m, cnt

    def magnetization(self, spins, mask, size) -> np.ndarray:
        s = np.ascontiguousarray(spins, dtype=np.float64)
        mm = np.ascontiguousarray(self.s.mu_s_muB(), dtype=np.float64)
        mk = np.ascontiguousarray(mask, dtype=np.int32)
        out = np.zeros(4 * size)
        lib().vref_magnetization(C.c_int(self.s.n), _p(mk, _I), C.c_int(size), _p(s[0], _D),
                                 _p(s[1], _D), _p(s[2], _D), _p(mm, _D), _p(out, _D))
        return out

    def energy(self, spins, mask, size) -> np.ndarray:
        s = np.ascontiguousarray(spins, dtype=np.float64)
        mm = np.ascontiguousarray(self.s.mu_s_muB(), dtype=np.float64)
        mk = np.ascontiguousarray(mask, dtype=np.int32)
        out = np.zeros(5 * size)
        lib().vref_energy(C.byref(self.st), _p(mk, _I), C.c_int(size), _p(s[0], _D), _p(s[1], _D),
                          _p(s[2], _D), _p(mm, _D), _p(out, _D))
        return out


# ----------------------------------------------------------------------------
# reference harness
# ----------------------------------------------------------------------------

def harness_available() -> bool:
    return HARNESS.exists()


def load_dump(d: Path) -> dict:
    out = {}
    for line in (Path(d) / "manifest.txt").read_text().splitlines():
        name, dt, cnt = line.split()
        out[name] = np.fromfile(Path(d) / f"{name}.bin", dtype=dt, count=int(cnt))
    return out


def run_harness(input_text: str, files: dict, args: list, workdir: Optional[str] = None,
                timeout: float = 600) -> dict:
    """Write `input` and material files into a scratch directory, run the
    reference harness there and return its dumped arrays."""
    if not harness_available():
        raise RuntimeError("reference harness not built (python oracle/build_ref.py)")
    tmp = workdir or tempfile.mkdtemp(prefix="vref_")
    Path(tmp, "input").write_text(input_text)
    for name, text in files.items():
        Path(tmp, name).write_text(text)
    out = Path(tmp, "out")
    out.mkdir(exist_ok=True)
    r = subprocess.run([str(HARNESS), "--out", str(out)] + [str(a) for a in args], cwd=tmp,
                       capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"harness failed rc={r.returncode}: {r.stdout[-2000:]} {r.stderr[-2000:]}")
    return load_dump(out)


def system_from_dump(d: dict, params=None):
    """Build a SpinSystem from a reference dump (harness --system)."""
    from vampire_b200 import system as S
    meta = d["meta"]
    n, nnz, nmat, et, uni, cub = [int(x) for x in meta[:6]]
    m16 = d["materials"].reshape(nmat, 16)
    mats = np.zeros(nmat, dtype=S.MATERIAL_DTYPE)
    for i in range(nmat):
        mats[i]["alpha"], mats[i]["gamma_rel"], mats[i]["mu_s_SI"] = m16[i, 0:3]
        mats[i]["one_oneplusalpha_sq"], mats[i]["alpha_oneplusalpha_sq"], mats[i]["H_th_sigma"] = m16[i, 3:6]
        mats[i]["temperature_rescaling_alpha"], mats[i]["temperature_rescaling_Tc"] = m16[i, 6:8]
        mats[i]["ku2"] = m16[i, 8]
        mats[i]["ku_vector"] = m16[i, 9:12]
        mats[i]["kc4"] = m16[i, 12]
        mats[i]["non_magnetic"] = int(m16[i, 13])
    simc = d["sim"]
    if params is None:
        params = S.SimParams(dt_SI=simc[2], gamma_SI=simc[3], temperature=simc[4], H_applied=simc[5],
                             H_vec=tuple(simc[6:9]), thermal=bool(meta[8]), applied=bool(meta[9]))
    if "sx_0" in d:
        spins = np.stack([d["sx_0"], d["sy_0"], d["sz_0"]])
    else:  # fixtures without a spin dump start along z
        spins = np.tile(np.array([[0.0], [0.0], [1.0]]), (1, n))
    s = S.SpinSystem(n=n, nl_start=d["nl_start"].astype(np.int32), nl_end=d["nl_end"].astype(np.int32),
                     nl=d["nl"].astype(np.int32), jlist=d["jlist"], exch_type=et,
                     type=d["type"].astype(np.int32), materials=mats, spins=spins, params=params,
                     uniaxial=bool(uni), cubic=bool(cub),
                     coords=np.stack([d["cx"], d["cy"], d["cz"]]))
    nt = d["nl_type"].astype(np.int32)
    if not np.array_equal(nt, np.arange(nt.size, dtype=np.int32)):
        s.nl_type = nt
    if "bq_flag" in d and int(d["bq_flag"][0]):
        s.biquadratic = {"start": d["bq_start"].astype(np.int32), "end": d["bq_end"].astype(np.int32),
                         "nl": d["bq_nl"].astype(np.int32), "type": d["bq_type"].astype(np.int32),
                         "jlist": d["bq_jlist"]}
    if "aniso_flags" in d and int(np.sum(d["aniso_flags"])) > 0:
        fl = [bool(x) for x in d["aniso_flags"]]
        ext = d["aniso_ext"].reshape(nmat, 12)
        s.aniso = {"u4": fl[0], "u6": fl[1], "c6": fl[2], "crot": fl[3], "neel": fl[4],
                   "ku4": ext[:, 0].copy(), "ku6": ext[:, 1].copy(), "kc6": ext[:, 2].copy(),
                   "kcb": ext[:, 3:12].copy(),
                   "neel_tensor": d["neel_tensor"].reshape(n, 9).copy() if fl[4] else None}
    if "mask_system" in d:
        s.masks["system"] = (d["mask_system"].astype(np.int32), int(d["sat_system"].size))
        s.masks["material"] = (d["mask_material"].astype(np.int32), int(d["sat_material"].size))
    return s
