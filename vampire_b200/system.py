"""Spin-system description in the reference's own data layout.

A :class:`SpinSystem` holds exactly what the reference keeps in its globals
and what ``vgpu_upload_system`` consumes (include/vgpu.h):

* the CSR neighbour list ``nl_start``/``nl_end`` (inclusive)/``nl`` of
  ``atoms::neighbour_list_*`` (src/exchange/initialize.cpp:70-117);
* the unrolled per-bond exchange list ``jlist`` in Tesla, 1, 3 or 9 doubles per
  bond (``atoms::i/v/t_exchange_list``, src/exchange/unroll_normalised.cpp:37-140);
* per-atom material ids and the per-material derived constants of
  ``set_derived_parameters`` (src/main/initialise_variables.cpp:352-432) and
  ``anisotropy::initialize`` (src/anisotropy/initialize.cpp:60-76).

Builders generate the synthetic lattices of the benchmark configurations
(simple-cubic and FCC boxes, spheres) with nearest-neighbour exchange and the
reference's three-site DMI construction (src/exchange/dmi.cpp:46-221).
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

# Physical constants exactly as the reference uses them
KB = 1.3806503e-23          # src/constants/constants.cpp:23
MU_B = 9.27400915e-24       # src/constants/constants.cpp:22
GAMMA_SI = 1.76e11          # mp::gamma_SI default (src/main/material.cpp)

EXCH_ISOTROPIC, EXCH_VECTORIAL, EXCH_TENSORIAL = 0, 1, 2

# Layout of vgpu_material (include/vgpu.h)
MATERIAL_DTYPE = np.dtype([
    ("alpha", "f8"), ("gamma_rel", "f8"), ("mu_s_SI", "f8"),
    ("one_oneplusalpha_sq", "f8"), ("alpha_oneplusalpha_sq", "f8"), ("H_th_sigma", "f8"),
    ("temperature_rescaling_alpha", "f8"), ("temperature_rescaling_Tc", "f8"),
    ("ku2", "f8"), ("ku_vector", "f8", (3,)), ("kc4", "f8"), ("temperature", "f8"),
    ("applied_field", "f8", (3,)), ("non_magnetic", "i4"), ("pad_", "i4"),
], align=True)


@dataclass
class Material:
    """Material inputs in SI units, as in a reference material file."""
    alpha: float = 1.0                       # damping-constant
    mu_s_muB: float = 1.72                   # atomic-spin-moment !muB
    gamma_rel: float = 1.0
    Ku: float = 0.0                          # second-order-uniaxial-anisotropy-constant [J/atom]
    ku_axis: Sequence[float] = (0.0, 0.0, 1.0)
    Kc: float = 0.0                          # fourth-order-cubic-anisotropy-constant [J/atom]
    temperature_rescaling_alpha: float = 1.0
    temperature_rescaling_Tc: float = 0.0
    non_magnetic: int = 0
    temperature: float = 0.0
    applied_field: Sequence[float] = (0.0, 0.0, 0.0)
    Ku4: float = 0.0                         # fourth-order-uniaxial-anisotropy-constant [J/atom]
    Ku6: float = 0.0                         # sixth-order-uniaxial-anisotropy-constant [J/atom]
    Kc6: float = 0.0                         # sixth-order-cubic-anisotropy-constant [J/atom]
    kc_axis1: Optional[Sequence[float]] = None   # cubic-anisotropy-direction-1 (rotated cubic basis)
    kc_axis2: Optional[Sequence[float]] = None   # cubic-anisotropy-direction-2

    @property
    def mu_s_SI(self) -> float:
        return self.mu_s_muB * MU_B


def anisotropy_ext(mats: Sequence[Material], n: int) -> Optional[dict]:
    """Higher-order anisotropy of `mats` in the reference's reduced form
    (anisotropy/initialize.cpp:60-120: K / mu_s, and the rotated cubic basis
    e1, e2, e3 = e1 x e2 normalised), or None when every term is off."""
    u4 = any(m.Ku4 != 0.0 for m in mats)
    u6 = any(m.Ku6 != 0.0 for m in mats)
    c6 = any(m.Kc6 != 0.0 for m in mats)
    crot = any(m.kc_axis1 is not None or m.kc_axis2 is not None for m in mats)
    if not (u4 or u6 or c6 or crot):
        return None
    M = len(mats)
    kcb = np.zeros((M, 9))
    for i, m in enumerate(mats):
        e1 = np.asarray(m.kc_axis1 if m.kc_axis1 is not None else (1.0, 0.0, 0.0), dtype=np.float64)
        e2 = np.asarray(m.kc_axis2 if m.kc_axis2 is not None else (0.0, 1.0, 0.0), dtype=np.float64)
        e1 = e1 / np.linalg.norm(e1)
        e2 = e2 / np.linalg.norm(e2)
        e3 = np.cross(e1, e2)
        e3 = e3 / np.linalg.norm(e3)
        kcb[i] = np.concatenate([e1, e2, e3])
    inv = np.array([1.0 / (m.mu_s_muB * MU_B) for m in mats])
    return {"u4": u4, "u6": u6, "c6": c6, "crot": crot, "neel": False,
            "ku4": np.array([m.Ku4 for m in mats]) * inv, "ku6": np.array([m.Ku6 for m in mats]) * inv,
            "kc6": np.array([m.Kc6 for m in mats]) * inv, "kcb": kcb, "neel_tensor": None}


def add_neel(s: SpinSystem, K_SI, bond_vec: np.ndarray, threshold: int) -> None:
    """Neel pair anisotropy on atoms with fewer than `threshold` neighbours
    (anisotropy/initialize_neel.cpp): T_i = sum_j K_ij/mu_s,i e_ij e_ij over
    the atom's neighbours.  bond_vec: (nnz, 3) i->j vectors of s.nl."""
    K = np.atleast_2d(np.asarray(K_SI, dtype=np.float64))
    deg = s.nl_end - s.nl_start + 1
    T = np.zeros((s.n, 9))
    mus = s.materials["mu_s_SI"]
    for i in np.flatnonzero(deg < threshold):
        mi = s.type[i]
        for b in range(s.nl_start[i], s.nl_end[i] + 1):
            e = bond_vec[b] / np.linalg.norm(bond_vec[b])
            kij = K[mi, s.type[s.nl[b]]] / mus[mi]
            T[i] += kij * np.outer(e, e).ravel()
    if s.aniso is None:
        s.aniso = {"u4": False, "u6": False, "c6": False, "crot": False, "neel": True,
                   "ku4": None, "ku6": None, "kc6": None, "kcb": None, "neel_tensor": T}
    else:
        s.aniso["neel"] = True
        s.aniso["neel_tensor"] = T


def derive_materials(mats: Sequence[Material], dt_SI: float, gamma_SI: float = GAMMA_SI) -> np.ndarray:
    """Per-material derived constants (initialise_variables.cpp:423-432,
    anisotropy/initialize.cpp:60-76)."""
    dt = dt_SI * gamma_SI
    out = np.zeros(len(mats), dtype=MATERIAL_DTYPE)
    for i, m in enumerate(mats):
        A = -m.gamma_rel / (1.0 + m.alpha * m.alpha)
        out[i]["alpha"] = m.alpha
        out[i]["gamma_rel"] = m.gamma_rel
        out[i]["mu_s_SI"] = m.mu_s_SI
        out[i]["one_oneplusalpha_sq"] = A
        out[i]["alpha_oneplusalpha_sq"] = m.alpha * A
        out[i]["H_th_sigma"] = np.sqrt(2.0 * m.alpha * KB / (m.mu_s_SI * m.gamma_rel * dt))
        out[i]["temperature_rescaling_alpha"] = m.temperature_rescaling_alpha
        out[i]["temperature_rescaling_Tc"] = m.temperature_rescaling_Tc
        inv_mu = 1.0 / (m.mu_s_muB * MU_B)
        out[i]["ku2"] = m.Ku * inv_mu
        out[i]["ku_vector"] = np.asarray(m.ku_axis, dtype=np.float64)
        out[i]["kc4"] = m.Kc * inv_mu
        out[i]["temperature"] = m.temperature
        out[i]["applied_field"] = np.asarray(m.applied_field, dtype=np.float64)
        out[i]["non_magnetic"] = m.non_magnetic
    return out


@dataclass
class SimParams:
    """Integration and field parameters (namespace sim / mp of the reference)."""
    dt_SI: float = 1.0e-16
    gamma_SI: float = GAMMA_SI
    temperature: float = 0.0
    H_applied: float = 0.0
    H_vec: Sequence[float] = (0.0, 0.0, 1.0)
    thermal: bool = True
    applied: bool = True
    local_temperature: bool = False
    local_applied_field: bool = False

    @property
    def dt(self) -> float:
        return self.dt_SI * self.gamma_SI

    @property
    def half_dt(self) -> float:
        return 0.5 * self.dt


@dataclass
class SpinSystem:
    n: int
    nl_start: np.ndarray
    nl_end: np.ndarray
    nl: np.ndarray
    jlist: np.ndarray
    exch_type: int
    type: np.ndarray
    materials: np.ndarray                      # MATERIAL_DTYPE records
    spins: np.ndarray                          # (3, n) float64
    params: SimParams = field(default_factory=SimParams)
    uniaxial: bool = False
    cubic: bool = False
    nl_type: Optional[np.ndarray] = None
    coords: Optional[np.ndarray] = None        # (3, n) Angstrom
    masks: dict = field(default_factory=dict)  # name -> (mask int32 [n], size)
    cells: Optional[dict] = None               # dipole macrocells (see dipole_cells())
    aniso: Optional[dict] = None               # higher-order anisotropy (see anisotropy_ext())
    bond_vectors: Optional[np.ndarray] = None  # (nnz, 3) i->j vectors [Angstrom] of the lattice builders
    biquadratic: Optional[dict] = None         # start, end, nl, type (or None), jlist [T]: biquadratic exchange

    @property
    def num_bonds(self) -> int:
        return int(self.nl.size)

    @property
    def num_materials(self) -> int:
        return int(self.materials.size)

    def mu_s_muB(self) -> np.ndarray:
        """atoms::m_spin_array: per-atom moment in Bohr magnetons."""
        return (self.materials["mu_s_SI"] / MU_B)[self.type]

    def sigma(self) -> np.ndarray:
        """Per-material thermal prefactor sqrt(T_rescaled) * H_th_sigma
        (src/simulate/fields.cpp:261-272)."""
        p = self.params
        out = np.zeros(self.num_materials)
        for m in range(self.num_materials):
            T = self.materials[m]["temperature"] if p.local_temperature else p.temperature
            a = self.materials[m]["temperature_rescaling_alpha"]
            Tc = self.materials[m]["temperature_rescaling_Tc"]
            Tr = Tc * (T / Tc) ** a if T < Tc else T
            out[m] = np.sqrt(Tr) * self.materials[m]["H_th_sigma"]
        return out

    def copy(self) -> "SpinSystem":
        import copy
        return copy.deepcopy(self)


# ----------------------------------------------------------------------------
# lattices
# ----------------------------------------------------------------------------

# basis in half-lattice-constant units and nearest-neighbour vectors
_BASIS = {
    "sc": np.array([[0, 0, 0]]),
    "fcc": np.array([[0, 0, 0], [1, 1, 0], [1, 0, 1], [0, 1, 1]]),
}
_NN = {
    "sc": np.array([[2, 0, 0], [-2, 0, 0], [0, 2, 0], [0, -2, 0], [0, 0, 2], [0, 0, -2]]),
    "fcc": np.array([[s1 * a, s2 * b, s3 * c]
                     for (a, b, c) in [(1, 1, 0), (1, 0, 1), (0, 1, 1)]
                     for s1 in (1, -1) for s2 in (1, -1) for s3 in (1, -1)
                     if not ((a == 0 and s1 < 0) or (b == 0 and s2 < 0) or (c == 0 and s3 < 0))]),
}


def lattice(kind: str, nx: int, ny: int, nz: int, a: float,
            periodic: Sequence[bool] = (True, True, True),
            keep: Optional[np.ndarray] = None):
    """Atoms of an nx*ny*nz box of `kind` ('sc'|'fcc') unit cells of size `a`
    [Angstrom] and their nearest-neighbour CSR.  Atom order: basis fastest,
    then x, y, z cells.  `keep` optionally masks atoms (e.g. a sphere) before
    numbering.  Returns (coords (3,n), nl_start, nl_end, nl, bond_vectors
    (nnz,3) in Angstrom)."""
    basis = _BASIS[kind]
    nnv = _NN[kind]
    nb = len(basis)
    cz, cy, cx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cells = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1)            # (ncell,3)
    half = (2 * cells[:, None, :] + basis[None, :, :]).reshape(-1, 3)         # (ncell*nb,3)
    full_n = half.shape[0]
    if keep is None:
        keep = np.ones(full_n, dtype=bool)
    idx = -np.ones(full_n, dtype=np.int64)
    idx[keep] = np.arange(int(keep.sum()))
    dims = np.array([2 * nx, 2 * ny, 2 * nz])
    grid = -np.ones((2 * nz, 2 * ny, 2 * nx), dtype=np.int64)
    grid[half[:, 2], half[:, 1], half[:, 0]] = idx
    hk = half[keep]
    n = hk.shape[0]
    nbrs = np.empty((n, len(nnv)), dtype=np.int64)
    for k, d in enumerate(nnv):
        q = hk + d
        valid = np.ones(n, dtype=bool)
        for ax in range(3):
            if periodic[ax]:
                q[:, ax] %= dims[ax]
            else:
                valid &= (q[:, ax] >= 0) & (q[:, ax] < dims[ax])
                q[:, ax] = np.clip(q[:, ax], 0, dims[ax] - 1)
        j = grid[q[:, 2], q[:, 1], q[:, 0]]
        nbrs[:, k] = np.where(valid, j, -1)
    valid = nbrs >= 0
    counts = valid.sum(axis=1)
    nl_start = np.zeros(n, dtype=np.int32)
    nl_start[1:] = np.cumsum(counts)[:-1]
    nl_end = (nl_start + counts - 1).astype(np.int32)
    nl = nbrs[valid].astype(np.int32)
    vec = np.broadcast_to(nnv[None, :, :], (n, len(nnv), 3))[valid].astype(np.float64) * (0.5 * a)
    coords = (hk.T.astype(np.float64)) * (0.5 * a)
    return coords, nl_start, nl_end, nl, vec


def exchange_lists(nl_start, nl_end, nl, types, materials: np.ndarray, Jmat_SI: np.ndarray,
                   exch_type: int = EXCH_ISOTROPIC) -> np.ndarray:
    """Unrolled per-bond exchange in Tesla: J_ij = Jmat_SI[mi][mj] / mu_s(mi)
    (unroll_normalised.cpp:37-140 with unit-cell J = 1)."""
    n = nl_start.size
    counts = (nl_end - nl_start + 1).astype(np.int64)
    ai = np.repeat(np.arange(n), counts)
    mi = types[ai]
    mj = types[nl]
    Jt = np.asarray(Jmat_SI, dtype=np.float64)[mi, mj] / materials["mu_s_SI"][mi]
    if exch_type == EXCH_ISOTROPIC:
        return Jt
    if exch_type == EXCH_VECTORIAL:
        return np.repeat(Jt[:, None], 3, axis=1).ravel()
    t = np.zeros((Jt.size, 3, 3))
    t[:, 0, 0] = Jt
    t[:, 1, 1] = Jt
    t[:, 2, 2] = Jt
    return t.reshape(-1)


def add_dmi(jlist9: np.ndarray, nl_start, nl_end, nl, bond_vec, types, materials: np.ndarray,
            dmi_SI: np.ndarray, cutoff: float = 2.6) -> np.ndarray:
    """Add the reference three-site DMI to a tensor exchange list
    (src/exchange/dmi.cpp:46-221): for bond i-j, sum over neighbours k of i
    (k != j) with |r_ik| and |r_jk| within `cutoff` [Angstrom] of
    D = 0.5 (dmi[mi][mk] + dmi[mj][mk]) / mu_s(i) times (e_ik x e_jk), stored
    as the antisymmetric tensor part J_xy -= D_z, J_xz += D_y, J_yx += D_z,
    J_yz -= D_x, J_zx -= D_y, J_zy += D_x.  Vectorised over atoms, looping
    over (j, k) neighbour slots; rows are padded to the maximum degree."""
    n = nl_start.size
    counts = (nl_end - nl_start + 1).astype(np.int64)
    zmax = int(counts.max()) if n else 0
    t = jlist9.reshape(-1, 3, 3).copy()
    dmi_SI = np.asarray(dmi_SI, dtype=np.float64)
    inv_mu = 1.0 / materials["mu_s_SI"]
    cut2 = cutoff * cutoff
    regular = (n > 0 and np.all(counts == zmax) and np.array_equal(nl_start, np.arange(n) * zmax))
    if regular:
        V = bond_vec.reshape(n, zmax, 3)
        if np.all(V.max(axis=0) - V.min(axis=0) == 0.0):
            # every atom sees the same neighbour vectors in the same order
            # (periodic lattice): D_ij direction is one constant per slot pair
            return _add_dmi_uniform(t, V[0], nl.reshape(n, zmax), types, dmi_SI, inv_mu, cut2).reshape(-1)
    # padded slot views
    slot_ok = np.arange(zmax)[None, :] < counts[:, None]
    bidx = np.where(slot_ok, nl_start[:, None] + np.arange(zmax)[None, :], 0)
    nbr = np.where(slot_ok, nl[bidx], 0)
    V = bond_vec[bidx]                                   # (n, zmax, 3)
    mi = types
    acc = np.zeros((n, zmax, 3, 3))
    for js in range(zmax):
        ok_j = slot_ok[:, js]
        mj = types[nbr[:, js]]
        eij = V[:, js, :]
        for ks in range(zmax):
            if ks == js:
                continue
            ok = ok_j & slot_ok[:, ks] & (nbr[:, ks] != nbr[:, js])
            eik = V[:, ks, :]
            ejk = eik - eij
            mik = (eik * eik).sum(1)
            mjk = (ejk * ejk).sum(1)
            ok &= (mik <= cut2) & (mjk <= cut2)
            if not ok.any():
                continue
            rows = np.nonzero(ok)[0]
            uik = eik[rows] / np.sqrt(mik[rows])[:, None]
            ujk = ejk[rows] / np.sqrt(mjk[rows])[:, None]
            mk = types[nbr[rows, ks]]
            Dij = 0.5 * (dmi_SI[mi[rows], mk] + dmi_SI[mj[rows], mk]) * inv_mu[mi[rows]]
            D = np.cross(uik, ujk)
            a = acc[rows, js]
            a[:, 0, 1] -= Dij * D[:, 2]
            a[:, 0, 2] -= Dij * -D[:, 1]
            a[:, 1, 0] -= Dij * -D[:, 2]
            a[:, 1, 2] -= Dij * D[:, 0]
            a[:, 2, 0] -= Dij * D[:, 1]
            a[:, 2, 1] -= Dij * -D[:, 0]
            acc[rows, js] = a
    t[bidx[slot_ok]] += acc[slot_ok]
    return t.reshape(-1)


def _add_dmi_uniform(t, v0, nbr, types, dmi_SI, inv_mu, cut2):
    """add_dmi for lattices where all atoms share the neighbour vectors v0
    (zmax, 3): same arithmetic, vectorised over atoms per (j, k) slot pair."""
    n, zmax = nbr.shape
    t = t.reshape(n, zmax, 3, 3)
    mi = types
    scale_i = inv_mu[mi]
    for js in range(zmax):
        mj = types[nbr[:, js]]
        eij = v0[js]
        for ks in range(zmax):
            if ks == js:
                continue
            eik = v0[ks]
            ejk = eik - eij
            mik = float((eik * eik).sum())
            mjk = float((ejk * ejk).sum())
            if not (mik <= cut2 and mjk <= cut2):
                continue
            uik = eik / np.sqrt(mik)
            ujk = ejk / np.sqrt(mjk)
            D = np.cross(uik, ujk)
            mk = types[nbr[:, ks]]
            ok = nbr[:, ks] != nbr[:, js]
            Dij = 0.5 * (dmi_SI[mi, mk] + dmi_SI[mj, mk]) * scale_i
            Dij = np.where(ok, Dij, 0.0)
            t[:, js, 0, 1] -= Dij * D[2]
            t[:, js, 0, 2] -= Dij * -D[1]
            t[:, js, 1, 0] -= Dij * -D[2]
            t[:, js, 1, 2] -= Dij * D[0]
            t[:, js, 2, 0] -= Dij * D[1]
            t[:, js, 2, 1] -= Dij * -D[0]
    return t


def random_spins(n: int, seed: int) -> np.ndarray:
    """Spins uniform on the unit sphere (normalised Gaussian triples)."""
    rng = np.random.default_rng(seed)
    s = rng.standard_normal((3, n))
    s /= np.sqrt((s * s).sum(0))
    return s


def build(kind: str, nx: int, ny: int, nz: int, a: float, mats: Sequence[Material],
          Jmat_SI, params: SimParams, *, periodic=(True, True, True), types=None,
          dmi_SI=None, dmi_cutoff: float = 2.6, exch_type: Optional[int] = None,
          keep=None, spin_seed: int = 123456, spins=None) -> SpinSystem:
    """Generate a SpinSystem of nearest-neighbour exchange on a lattice."""
    coords, st, en, nl, vec = lattice(kind, nx, ny, nz, a, periodic, keep)
    n = coords.shape[1]
    materials = derive_materials(mats, params.dt_SI, params.gamma_SI)
    if types is None:
        types = np.zeros(n, dtype=np.int32)
    types = np.asarray(types, dtype=np.int32)
    Jmat = np.atleast_2d(np.asarray(Jmat_SI, dtype=np.float64))
    if exch_type is None:
        exch_type = EXCH_TENSORIAL if dmi_SI is not None else EXCH_ISOTROPIC
    jl = exchange_lists(st, en, nl, types, materials, Jmat, exch_type)
    if dmi_SI is not None:
        jl = add_dmi(jl, st, en, nl, vec, types, materials, np.atleast_2d(dmi_SI), dmi_cutoff)
    if spins is None:
        spins = random_spins(n, spin_seed)
    ext = anisotropy_ext(mats, n)
    rotated = ext is not None and ext["crot"]
    sys_ = SpinSystem(n=n, nl_start=st, nl_end=en, nl=nl, jlist=jl, exch_type=exch_type,
                      type=types, materials=materials, spins=np.ascontiguousarray(spins),
                      params=params, uniaxial=any(m.Ku != 0.0 for m in mats),
                      cubic=any(m.Kc != 0.0 for m in mats) and not rotated, coords=coords, aniso=ext)
    sys_.masks["system"] = (np.zeros(n, dtype=np.int32), 1)
    sys_.masks["material"] = (types.copy(), len(mats))
    sys_.bond_vectors = vec
    return sys_


def dipole_cells(s: SpinSystem, size: float, atomic_volume: float, solver: str = "tensor",
                 cutoff: float = 2.0, update_rate: int = 100) -> dict:
    """Macrocells of edge `size` [Angstrom] on a regular grid from the atom
    positions, as cells::initialize builds them (src/cells/initialize.cpp:
    moment-weighted centres, volume = atoms x atomic volume).  Stored in
    s.cells and returned (the dict vgpu.Simulation.dipole_setup takes)."""
    c = s.coords
    lo = c.min(axis=1)
    idx = np.floor((c - lo[:, None]) / size + 1e-9).astype(np.int64)
    dims = idx.max(axis=1) + 1
    cell = (idx[0] + dims[0] * (idx[1] + dims[1] * idx[2])).astype(np.int32)
    nc = int(np.prod(dims))
    mu = s.materials["mu_s_SI"][s.type]
    magnetic = s.materials["non_magnetic"][s.type] == 0
    w = np.where(magnetic, mu, 0.0)
    natoms = np.bincount(cell, weights=magnetic.astype(np.float64), minlength=nc).astype(np.int32)
    pm = np.zeros((nc, 4))
    for q in range(3):
        pm[:, q] = np.bincount(cell, weights=c[q] * w, minlength=nc)
    pm[:, 3] = np.bincount(cell, weights=w, minlength=nc)
    has = pm[:, 3] > 0
    pm[has, :3] /= pm[has, 3:4]
    vol = natoms * atomic_volume
    s.cells = {"atom_cell": cell, "cell_pos_mom": pm.ravel(), "cell_volume": vol.astype(np.float64),
               "cell_natoms": natoms, "macro_cell_size": size, "cutoff": cutoff, "update_rate": update_rate,
               "solver": solver, "coords": s.coords}
    return s.cells


def replicas(s: SpinSystem, temperatures: Sequence[float]) -> SpinSystem:
    """len(temperatures) independent copies of `s` in one system (temperature
    replicas): copy k uses materials k*M..k*M+M-1, identical to s's except for
    their temperature, and local temperatures are switched on.  Masks:
    "replica" (bin k) and "material" (bin k*M+m)."""
    k = len(temperatures)
    M = s.num_materials
    if k * M > 100:
        raise ValueError("at most 100 materials (replicas x materials) per handle")
    n, nb = s.n, s.num_bonds
    mats = np.concatenate([s.materials.copy() for _ in range(k)])
    for r, T in enumerate(temperatures):
        mats["temperature"][r * M:(r + 1) * M] = T
    off = np.repeat(np.arange(k, dtype=np.int64) * n, n)
    boff = np.repeat(np.arange(k, dtype=np.int64) * nb, n)
    st = (np.tile(s.nl_start.astype(np.int64), k) + boff).astype(np.int32)
    en = (np.tile(s.nl_end.astype(np.int64), k) + boff).astype(np.int32)
    nl = (np.tile(s.nl.astype(np.int64), k) + np.repeat(np.arange(k, dtype=np.int64) * n, nb)).astype(np.int32)
    if s.nl_type is not None:
        nl_type, jl = np.tile(s.nl_type, k), s.jlist
    else:
        nl_type, jl = None, np.tile(s.jlist, k)
    typ = (np.tile(s.type, k) + np.repeat(np.arange(k) * M, n)).astype(np.int32)
    p = dataclasses.replace(s.params, local_temperature=True)
    out = SpinSystem(n=k * n, nl_start=st, nl_end=en, nl=nl, jlist=jl, exch_type=s.exch_type, type=typ,
                     materials=mats, spins=np.tile(s.spins, (1, k)), params=p, uniaxial=s.uniaxial, cubic=s.cubic,
                     nl_type=nl_type, coords=None)
    if s.aniso is not None:
        a = dict(s.aniso)
        for key in ("ku4", "ku6", "kc6"):
            if a[key] is not None:
                a[key] = np.tile(a[key], k)
        if a["kcb"] is not None:
            a["kcb"] = np.tile(a["kcb"], (k, 1))
        if a["neel_tensor"] is not None:
            a["neel_tensor"] = np.tile(a["neel_tensor"], (k, 1))
        out.aniso = a
    out.masks["system"] = (np.zeros(k * n, dtype=np.int32), 1)
    out.masks["replica"] = ((off // n).astype(np.int32), k)
    out.masks["material"] = (typ.copy(), k * M)
    return out


# ----------------------------------------------------------------------------
# benchmark configurations (synthetic inputs with the configurations' shapes)
# ----------------------------------------------------------------------------

def config_sc_llg(L: int = 20, temperature: float = 0.0, seed: int = 123456) -> SpinSystem:
    """Simple-cubic ferromagnet, L^3 periodic, a=0.3 nm, J=11.2e-21 J (6 nn),
    Ku=6.69e-24 J/atom along z, mu_s=1.72 muB, alpha=0.1, dt=1e-16 s,
    H=(0,0,0.1) T; spins uniform on the sphere."""
    m = Material(alpha=0.1, mu_s_muB=1.72, Ku=6.69e-24)
    p = SimParams(dt_SI=1e-16, temperature=temperature, H_applied=0.1, H_vec=(0.0, 0.0, 1.0))
    return build("sc", L, L, L, 3.0, [m], [[11.2e-21]], p, spin_seed=seed)


def config_fcc_tensor(L: int = 100, seed: int = 2024, temperature: float = 300.0,
                      dipole: bool = False, periodic=(True, True, True)) -> SpinSystem:
    """FCC L^3 periodic (4 L^3 spins), a=0.354 nm, two materials at random
    50/50, nn tensor exchange J_AA=J_BB=11.2e-21 J, J_AB=5e-21 J plus the
    three-site DMI with D=0.1 J, cubic Kc=1e-24 J/atom, alpha=0.05,
    dt=1e-16 s, T=300 K, H=0; with `dipole`, 2x2x2-unit-cell macrocells;
    `periodic` per axis (open surfaces give atoms fewer than 12 bonds)."""
    mats = [Material(alpha=0.05, mu_s_muB=1.72, Kc=1e-24) for _ in range(2)]
    J = np.array([[11.2e-21, 5e-21], [5e-21, 11.2e-21]])
    p = SimParams(dt_SI=1e-16, temperature=temperature, H_applied=0.0, H_vec=(0.0, 0.0, 1.0))
    rng = np.random.default_rng(seed)
    types = (rng.random(4 * L ** 3) < 0.5).astype(np.int32)
    s = build("fcc", L, L, L, 3.54, mats, J, p, periodic=tuple(periodic), types=types, dmi_SI=0.1 * J,
              spin_seed=seed + 1)
    if dipole:
        # macrocells of 2x2x2 unit cells, tensor solver, updated every 100 steps
        dipole_cells(s, size=2 * 3.54, atomic_volume=3.54 ** 3 / 4.0, solver="tensor", update_rate=100)
    return s
