"""Generate the golden fixtures in tests/golden/ from the reference program.

Needs the reference harness (python oracle/build_ref.py, which compiles the
reference sources in place).  Each fixture is an .npz holding what the
reference itself built and produced: its CSR neighbour list, unrolled exchange
list, material constants, initial spins, spins after N of its own
sim::LLG_Heun() steps, the Gaussian stream it consumed (captured by the
harness through MTRand get_state/set_state) and its statistics.

    python tests/golden/make_golden.py            # all fixtures
    python tests/golden/make_golden.py sc10_t300  # one
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import oracle as O  # noqa: E402
from oracle.refinputs import SC_MAT, fcc_input, fcc_mat, sc_input  # noqa: E402


SYSTEM_KEYS = ["meta", "nl_start", "nl_end", "nl", "nl_type", "type", "m_spin", "cx", "cy", "cz", "jlist",
               "materials", "sim", "mask_system", "sat_system", "mask_material", "sat_material",
               "aniso_flags", "aniso_ext", "neel_tensor"]


def save(name: str, d: dict, keep: list) -> None:
    out = {k: d[k] for k in SYSTEM_KEYS if k in d}
    for k in keep:
        out[k] = d[k]
    # per-bond exchange of a regular lattice is highly repetitive; npz-compress everything
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(f"{name}: {sum(v.nbytes for v in out.values()) / 1e6:.2f} MB raw")


def sc20_t0():
    """Config-0 system (SC 20^3 periodic), T=0: the reference trajectory at
    steps 1, 100 and 10,000 (deterministic check)."""
    d = O.run_harness(sc_input(20), {"m.mat": SC_MAT},
                      ["--system", "--steps", 10000, "--snaps", "1,100,10000", "--stats", "0,10000"])
    keep = [f"s{c}_{t}" for t in (0, 1, 100, 10000) for c in "xyz"]
    keep += ["mag_system_0", "energy_system_0", "mag_system_10000", "energy_system_10000",
             "mag_material_10000", "energy_material_10000"]
    save("sc20_t0", d, keep)


def sc8_t0():
    """SC 8^3 periodic at T=0: reference spins at many steps (fast checks)."""
    d = O.run_harness(sc_input(8), {"m.mat": SC_MAT},
                      ["--system", "--steps", 2000, "--snaps", "1,2,10,100,1000,2000"])
    keep = [f"s{c}_{t}" for t in (0, 1, 2, 10, 100, 1000, 2000) for c in "xyz"]
    save("sc8_t0", d, keep)


def sc10_t300():
    """SC 10^3 periodic at T=300 K: one and two replayed stochastic steps."""
    d = O.run_harness(sc_input(10, T=300.0), {"m.mat": SC_MAT},
                      ["--system", "--steps", 2, "--snaps", "1,2", "--noise", 2])
    keep = [f"s{c}_{t}" for t in (0, 1, 2) for c in "xyz"] + ["xi_1", "xi_2"]
    save("sc10_t300", d, keep)


def sc6_open_t300():
    """SC 6^3 with open boundaries (ragged CSR rows) at T=300 K, replayed noise."""
    d = O.run_harness(sc_input(6, T=300.0, periodic=False), {"m.mat": SC_MAT},
                      ["--system", "--steps", 3, "--snaps", "1,3", "--noise", 3, "--stats", "3"])
    keep = [f"s{c}_{t}" for t in (0, 1, 3) for c in "xyz"] + ["xi_1", "xi_2", "xi_3",
                                                              "mag_system_3", "energy_system_3"]
    save("sc6_open_t300", d, keep)


def fcc4_dmi_t300():
    """FCC 4^3 periodic random A/B alloy, nn tensor exchange + three-site DMI +
    cubic anisotropy, T=300 K: one replayed step, plus stats."""
    d = O.run_harness(fcc_input(4, T=300.0), {"m.mat": fcc_mat()},
                      ["--system", "--steps", 2, "--snaps", "1,2", "--noise", 2, "--stats", "0,2"])
    keep = [f"s{c}_{t}" for t in (0, 1, 2) for c in "xyz"] + ["xi_1", "xi_2", "mag_system_2",
                                                              "energy_system_2", "mag_material_2",
                                                              "energy_material_2"]
    save("fcc4_dmi_t300", d, keep)


def fcc4_dmi_t0():
    """Same FCC alloy at T=0: 200 deterministic steps."""
    d = O.run_harness(fcc_input(4, T=0.0), {"m.mat": fcc_mat()},
                      ["--system", "--steps", 200, "--snaps", "1,200"])
    keep = [f"s{c}_{t}" for t in (0, 1, 200) for c in "xyz"]
    save("fcc4_dmi_t0", d, keep)


def single_spin_applied():
    """The reference's own known-answer setup (tests/physical/AppliedField):
    one spin along x, H=10 T along z, alpha=1, T=0, dt=1e-16 s."""
    inp = ("create:single-spin\nmaterial:file=m.mat\nsim:temperature=0.0\nsim:time-step=1.0E-16\n"
           "sim:applied-field-strength=10.0 !T\nsim:applied-field-unit-vector=0,0,1\n"
           "sim:program=time-series\nsim:integrator=llg-heun\n")
    mat = ("material:num-materials=1\nmaterial[1]:material-name=Co\nmaterial[1]:damping-constant=1\n"
           "material[1]:exchange-matrix[1]=11.2e-21\nmaterial[1]:atomic-spin-moment=1.72 !muB\n"
           "material[1]:uniaxial-anisotropy-constant=0.0\nmaterial[1]:initial-spin-direction=1,0,0\n")
    d = O.run_harness(inp, {"m.mat": mat}, ["--system", "--steps", 10000, "--snaps", "50,1000,5000,10000"])
    keep = [f"s{c}_{t}" for t in (0, 50, 1000, 5000, 10000) for c in "xyz"]
    save("single_spin_applied", d, keep)


def sc6_derived_t600():
    """SC 6^3 periodic at T=600 K: 20 stochastic steps (Gaussian stream
    replayed), statistics after every step, and the reference's derived
    statistics (susceptibility, specific heat, standard deviation)."""
    d = O.run_harness(sc_input(6, T=600.0), {"m.mat": SC_MAT},
                      ["--system", "--steps", 20, "--noise", 20, "--stats-every", 1, "--derived", "--snaps", "20"])
    keep = [f"s{c}_{t}" for t in (0, 20) for c in "xyz"] + [f"xi_{t}" for t in range(1, 21)]
    keep += ["sus_system", "sus_material", "spec_heat_system", "spec_heat_material", "std_material"]
    save("sc6_derived_t600", d, keep)


def sc8_midpoint():
    """The LLG-Midpoint integrator (sim:integrator=llg-midpoint,
    src/simulate/LLGMidpoint.cpp) on SC 8^3 periodic: 100 deterministic steps
    at T=0, and 2 stochastic steps at T=300 K with the Gaussian stream."""
    d = O.run_harness(sc_input(8, integrator="llg-midpoint"), {"m.mat": SC_MAT},
                      ["--system", "--steps", 100, "--snaps", "1,100"])
    keep = [f"s{c}_{t}" for t in (0, 1, 100) for c in "xyz"]
    save("sc8_midpoint_t0", d, keep)
    d = O.run_harness(sc_input(8, T=300.0, integrator="llg-midpoint"), {"m.mat": SC_MAT},
                      ["--system", "--steps", 2, "--snaps", "1,2", "--noise", 2])
    keep = [f"s{c}_{t}" for t in (0, 1, 2) for c in "xyz"] + ["xi_1", "xi_2"]
    save("sc8_midpoint_t300", d, keep)


BQ_MAT = SC_MAT.replace("material[1]:exchange-matrix[1]=11.2e-21\n",
                        "material[1]:exchange-matrix[1]=11.2e-21\nmaterial[1]:biquadratic-exchange[1]=2.0e-21\n")


def sc6_biquadratic():
    """SC 6^3, open boundaries, biquadratic exchange (material
    biquadratic-exchange, src/exchange/biquadratic_fields.cpp) on top of the
    bilinear exchange and uniaxial anisotropy: 200 T=0 reference steps and
    energies, and 2 stochastic steps at 300 K with the Gaussian stream."""
    d = O.run_harness(sc_input(6, periodic=False), {"m.mat": BQ_MAT},
                      ["--system", "--steps", 200, "--snaps", "1,200", "--stats", "0,200"])
    keep = [f"s{c}_{t}" for t in (0, 1, 200) for c in "xyz"]
    keep += ["mag_system_0", "energy_system_0", "mag_system_200", "energy_system_200",
             "bq_flag", "bq_start", "bq_end", "bq_nl", "bq_type", "bq_jlist"]
    save("sc6_biquadratic_t0", d, keep)
    d = O.run_harness(sc_input(6, T=300.0, periodic=False), {"m.mat": BQ_MAT},
                      ["--system", "--steps", 2, "--snaps", "1,2", "--noise", 2])
    keep = [f"s{c}_{t}" for t in (0, 1, 2) for c in "xyz"] + ["xi_1", "xi_2", "bq_flag", "bq_start", "bq_end",
                                                              "bq_nl", "bq_type", "bq_jlist"]
    save("sc6_biquadratic_t300", d, keep)


HO_MAT = """material:num-materials=1
material[1]:material-name=A
material[1]:damping-constant=0.1
material[1]:exchange-matrix[1]=11.2e-21
material[1]:atomic-spin-moment=1.72 !muB
material[1]:second-order-uniaxial-anisotropy-constant=6.69e-24
material[1]:fourth-order-uniaxial-anisotropy-constant=2.0e-24
material[1]:sixth-order-uniaxial-anisotropy-constant=1.0e-24
material[1]:fourth-order-cubic-anisotropy-constant=1.0e-24
material[1]:sixth-order-cubic-anisotropy-constant=3.0e-24
material[1]:uniaxial-anisotropy-direction=0,0.6,0.8
material[1]:initial-spin-direction=random
"""


def sc6_aniso_ho():
    """SC 6^3, open boundaries, T=0: second-, fourth- and sixth-order uniaxial
    anisotropy along (0, 0.6, 0.8) plus fourth- and sixth-order cubic
    anisotropy; 200 reference steps and energies."""
    d = O.run_harness(sc_input(6, periodic=False), {"m.mat": HO_MAT},
                      ["--system", "--steps", 200, "--snaps", "1,200", "--stats", "0,200"])
    keep = [f"s{c}_{t}" for t in (0, 1, 200) for c in "xyz"]
    keep += ["mag_system_0", "energy_system_0", "energy_material_0", "mag_system_200", "energy_system_200"]
    save("sc6_aniso_ho", d, keep)


def fcc4_neel_rot():
    """FCC 4^3 cube, open boundaries: rotated cubic anisotropy (axes [110],
    [-110], [001]) and Neel surface anisotropy on atoms with fewer than 12
    neighbours; T=0, 100 reference steps and energies."""
    a, L = 3.54, 4
    size = L * a / 10.0
    inp = (f"create:crystal-structure=fcc\ndimensions:unit-cell-size={a} !A\n"
           f"dimensions:system-size-x={size} !nm\ndimensions:system-size-y={size} !nm\n"
           f"dimensions:system-size-z={size} !nm\nmaterial:file=m.mat\nsim:temperature=0.0\n"
           f"sim:time-step=1.0E-16\nsim:program=time-series\nsim:integrator=llg-heun\n"
           f"anisotropy:surface-anisotropy-threshold=12\n")
    mat = ("material:num-materials=1\nmaterial[1]:material-name=A\nmaterial[1]:damping-constant=0.1\n"
           "material[1]:exchange-matrix[1]=11.2e-21\nmaterial[1]:atomic-spin-moment=1.72 !muB\n"
           "material[1]:fourth-order-cubic-anisotropy-constant=1.0e-24\n"
           "material[1]:cubic-anisotropy-direction-1=1,1,0\nmaterial[1]:cubic-anisotropy-direction-2=-1,1,0\n"
           "material[1]:neel-anisotropy-constant[1]=5.0e-23\nmaterial[1]:initial-spin-direction=random\n")
    d = O.run_harness(inp, {"m.mat": mat}, ["--system", "--steps", 100, "--snaps", "1,100", "--stats", "0,100"])
    keep = [f"s{c}_{t}" for t in (0, 1, 100) for c in "xyz"]
    keep += ["mag_system_0", "energy_system_0", "energy_material_0", "mag_system_100", "energy_system_100"]
    save("fcc4_neel_rot", d, keep)


DIPOLE_KEYS = ["cell_id", "cell_natoms", "cell_volume", "cell_pos_mom"]


def _dipole_fixture(name: str, solver: str):
    """FCC 10^3 periodic A/B alloy (tensor exchange + DMI + cubic) with
    2x2x2-unit-cell macrocells (7.08 A), reference dipole solver `solver`,
    T=0: cell moments and fields at start-up, and the reference trajectory
    across the field update at step 100."""
    extra = f"cells:macro-cell-size=7.08 !A\ndipole:solver={solver}\ndipole:field-update-rate=100\n"
    d = O.run_harness(fcc_input(10, T=0.0, extra=extra), {"m.mat": fcc_mat()},
                      ["--system", "--steps", 101, "--snaps", "99,100,101", "--dipole"])
    keep = DIPOLE_KEYS + [f"s{c}_{t}" for t in (0, 99, 100, 101) for c in "xyz"]
    keep += [f"{q}_{c}_{t}" for q in ("cmag", "cfield", "chd") for c in "xyz" for t in (0, 100)]
    save(name, d, keep)


def fcc10_dipole_tensor():
    _dipole_fixture("fcc10_dipole_tensor", "tensor")


def fcc10_dipole_macrocell():
    _dipole_fixture("fcc10_dipole_macrocell", "macrocell")


MC_MAT = SC_MAT.replace("initial-spin-direction=random", "initial-spin-direction=0,0,1")
MC_TEMPS = [50.0 * k for k in range(31)]
MC_EQ, MC_AV, MC_EVERY = 2000, 20000, 10


def _mc_one(T):
    inp = sc_input(16, T=T, H=0.0, integrator="monte-carlo", extra="montecarlo:algorithm=angle\n")
    d = O.run_harness(inp, {"m.mat": MC_MAT}, ["--system", "--steps", MC_EQ + MC_AV, "--mag-every", MC_EVERY,
                                               "--mag-start", MC_EQ], timeout=3600)
    return d


def blocking_stats(x: np.ndarray, nblocks: int = 10):
    """Mean and standard error of a correlated series from block means."""
    x = np.asarray(x)
    b = x[: len(x) // nblocks * nblocks].reshape(nblocks, -1).mean(1)
    return float(x.mean()), float(b.std(ddof=1) / np.sqrt(nblocks))


def mc_sc16_curie():
    """Reference Metropolis Curie sweep (sequential random-site angle moves,
    montecarlo::mc_step): SC 16^3 periodic, config-0 material, H=0, spins
    start along z, 31 temperatures 0..1500 K, 2000 equilibration + 20000
    averaging sweeps, |m| sampled every 10 sweeps, standard errors from 10
    blocks of 2000 sweeps.  Independent processes,
    one per temperature."""
    from concurrent.futures import ThreadPoolExecutor
    import os
    with ThreadPoolExecutor(os.cpu_count() or 4) as ex:
        runs = list(ex.map(_mc_one, MC_TEMPS))
    mean, se, acc = [], [], []
    for d in runs:
        tr = d["mag_trace"].reshape(-1, 4)[:, 3]
        m, e = blocking_stats(tr)
        mean.append(m)
        se.append(e)
        mv, rj = d["mc_counters"]
        acc.append(1.0 - rj / mv)
    d0 = runs[0]
    out = {k: d0[k] for k in SYSTEM_KEYS if k in d0}
    out.update(T=np.array(MC_TEMPS), m_mean=np.array(mean), m_se=np.array(se), acceptance=np.array(acc),
               sweeps=np.array([MC_EQ, MC_AV, MC_EVERY]))
    np.savez_compressed(HERE / "mc_sc16_curie.npz", **out)
    print("mc_sc16_curie:", np.round(mean, 3))


def _tet_ucf(kind: str) -> str:
    """Unit-cell file (the reference's .ucf format, src/unitcell/read.cpp and
    read_interactions.cpp) of a two-atom tetragonal cell, 3 x 3 x 6 A: atom 0
    (material 1) at the origin, atom 1 (material 2) at z = 1/2, bonds along
    +-x and +-y to the same sublattice and along +-z to the other.  Every
    bond direction has its own coupling, so no coupling is a function of the
    two materials alone: the reference holds it per bond.  kind: isotropic
    (1 value per bond), vectorial (3) or tensorial (9, with J_ji = J_ij^T and
    off-diagonal symmetric and antisymmetric parts)."""
    rng = np.random.default_rng({"isotropic": 1, "vectorial": 2, "tensorial": 3}[kind])
    bonds = []  # (i, j, dx, dy, dz, key, transpose)
    for i in (0, 1):
        for sgn in (1, -1):
            bonds.append((i, i, sgn, 0, 0, ("x", i), sgn < 0))
            bonds.append((i, i, 0, sgn, 0, ("y", i), sgn < 0))
    bonds += [(0, 1, 0, 0, 0, ("z", 0), False), (1, 0, 0, 0, 0, ("z", 0), True),
              (0, 1, 0, 0, -1, ("z", 1), False), (1, 0, 0, 0, 1, ("z", 1), True)]
    base = {("x", 0): 11.2, ("y", 0): 8.0, ("x", 1): 6.0, ("y", 1): 13.0, ("z", 0): 10.0, ("z", 1): 4.0}
    mats = {}
    for key, j in base.items():
        m = np.diag(j * (1.0 + 0.25 * rng.uniform(-1, 1, 3))) if kind != "isotropic" else np.eye(3) * j
        if kind == "tensorial":
            a = 0.15 * j * rng.uniform(-1, 1, (3, 3))
            m = m + 0.5 * (a + a.T) + 0.5 * (a - a.T) * 0.8
        mats[key] = m * 1e-21
    lines = ["# Unit cell size:", "3.0 3.0 6.0", "# Unit cell vectors:", "1.0 0.0 0.0", "0.0 1.0 0.0",
             "0.0 0.0 1.0", "# Atoms num, id cx cy cz mat lc hc", "2", "0 0.0 0.0 0.0 0 0 0",
             "1 0.0 0.0 0.5 1 0 1", "# Interactions n exctype, id i j dx dy dz Jij", f"{len(bonds)} {kind}"]
    for n, (i, j, dx, dy, dz, key, tr) in enumerate(bonds):
        m = mats[key].T if tr else mats[key]
        if kind == "isotropic":
            vals = [m[0, 0]]
        elif kind == "vectorial":
            vals = [m[0, 0], m[1, 1], m[2, 2]]
        else:
            vals = list(m.reshape(-1))
        lines.append(f"{n} {i} {j} {dx} {dy} {dz} " + " ".join(f"{v:.17g}" for v in vals))
    return "\n".join(lines) + "\n"


TET_MAT = """material:num-materials=2
material[1]:material-name=A
material[1]:damping-constant=0.1
material[1]:exchange-matrix[1]=11.2e-21
material[1]:exchange-matrix[2]=10.0e-21
material[1]:atomic-spin-moment=1.72 !muB
material[1]:second-order-uniaxial-anisotropy-constant=6.69e-24
material[1]:uniaxial-anisotropy-direction=0,0,1
material[1]:initial-spin-direction=random
material[2]:material-name=B
material[2]:damping-constant=0.05
material[2]:exchange-matrix[1]=10.0e-21
material[2]:exchange-matrix[2]=11.2e-21
material[2]:atomic-spin-moment=2.2 !muB
material[2]:second-order-uniaxial-anisotropy-constant=3.0e-24
material[2]:uniaxial-anisotropy-direction=0,0.6,0.8
material[2]:initial-spin-direction=random
"""


def _tet_input(T: float) -> str:
    return ("material:unit-cell-file=cell.ucf\n" + "".join(f"create:periodic-boundaries-{c}\n" for c in "xyz") +
            "dimensions:system-size-x=1.8 !nm\ndimensions:system-size-y=1.8 !nm\n"
            "dimensions:system-size-z=1.8 !nm\nmaterial:file=m.mat\n"
            f"sim:temperature={T}\nsim:time-step=1.0E-16\nsim:applied-field-strength=0.1 !T\n"
            "sim:applied-field-unit-vector=0,0,1\nsim:program=time-series\nsim:integrator=llg-heun\n")


def _tet_bond(kind: str):
    files = {"m.mat": TET_MAT, "cell.ucf": _tet_ucf(kind)}
    d = O.run_harness(_tet_input(0.0), files, ["--system", "--steps", 200, "--snaps", "1,100,200", "--stats", "0,200"])
    keep = [f"s{c}_{t}" for t in (0, 1, 100, 200) for c in "xyz"]
    keep += ["mag_system_0", "energy_system_0", "mag_system_200", "energy_system_200", "mag_material_200",
             "energy_material_200"]
    save(f"tet_{kind[:3]}_bond_t0", d, keep)
    d = O.run_harness(_tet_input(300.0), files, ["--system", "--steps", 2, "--snaps", "1,2", "--noise", 2])
    keep = [f"s{c}_{t}" for t in (0, 1, 2) for c in "xyz"] + ["xi_1", "xi_2"]
    save(f"tet_{kind[:3]}_bond_t300", d, keep)


def tet_bond_exchange():
    """Per-bond exchange from a unit-cell file (the reference's non-normalised
    'isotropic', 'vectorial' and 'tensorial' interaction types,
    src/exchange/unroll.cpp:52-105): tetragonal two-material cell, 6 x 6 x 3
    cells (216 atoms), periodic, H = 0.1 T; 200 T=0 reference steps with
    energies, and 2 stochastic steps at 300 K with the Gaussian stream."""
    for kind in ("isotropic", "vectorial", "tensorial"):
        _tet_bond(kind)


VEC_MAT = SC_MAT.replace("material[1]:exchange-matrix[1]=11.2e-21\n",
                         "material[1]:exchange-matrix[1]=11.2e-21,8.0e-21,14.0e-21\n")


def sc6_vec():
    """Vectorial exchange from the material file (exchange-matrix with three
    values: the normalised vectorial form, src/exchange/interface.cpp:86-94,
    exchange_fields.cpp:82-117) on SC 6^3 periodic: 200 T=0 reference steps
    with energies, and 2 stochastic steps at 300 K with the Gaussian stream."""
    d = O.run_harness(sc_input(6), {"m.mat": VEC_MAT},
                      ["--system", "--steps", 200, "--snaps", "1,100,200", "--stats", "0,200"])
    keep = [f"s{c}_{t}" for t in (0, 1, 100, 200) for c in "xyz"]
    keep += ["mag_system_0", "energy_system_0", "mag_system_200", "energy_system_200"]
    save("sc6_vec_t0", d, keep)
    d = O.run_harness(sc_input(6, T=300.0), {"m.mat": VEC_MAT}, ["--system", "--steps", 2, "--snaps", "1,2", "--noise", 2])
    keep = [f"s{c}_{t}" for t in (0, 1, 2) for c in "xyz"] + ["xi_1", "xi_2"]
    save("sc6_vec_t300", d, keep)


def torque_fixtures():
    """Torque statistics (stats::system_torque, stats::max_torque,
    src/utility/statistics.cpp:221-325) at T=0: torque_<step> = system
    torque, per-material torque (x, y, z blocks), max |S x H|.  FCC 4^3 A/B
    alloy with tensor exchange + DMI + cubic anisotropy at steps 0 and 50;
    the per-bond tensorial tetragonal cell at steps 0 and 50; FCC 10^3 with
    the macrocell dipole field at step 0 (fields of the start-up update)."""
    d = O.run_harness(fcc_input(4, T=0.0), {"m.mat": fcc_mat()},
                      ["--system", "--steps", 50, "--snaps", "50", "--torque", "0,50"])
    save("torque_fcc4_t0", d, [f"s{c}_{t}" for t in (0, 50) for c in "xyz"] + ["torque_0", "torque_50"])
    files = {"m.mat": TET_MAT, "cell.ucf": _tet_ucf("tensorial")}
    d = O.run_harness(_tet_input(0.0), files, ["--system", "--steps", 50, "--snaps", "50", "--torque", "0,50"])
    save("torque_tet_t0", d, [f"s{c}_{t}" for t in (0, 50) for c in "xyz"] + ["torque_0", "torque_50"])
    extra = "cells:macro-cell-size=7.08 !A\ndipole:solver=macrocell\ndipole:field-update-rate=100\n"
    d = O.run_harness(fcc_input(10, T=0.0, extra=extra), {"m.mat": fcc_mat()},
                      ["--system", "--steps", 0, "--dipole", "--torque", "0"])
    keep = DIPOLE_KEYS + [f"s{c}_0" for c in "xyz"] + ["torque_0"]
    keep += [f"{q}_{c}_0" for q in ("cmag", "cfield", "chd") for c in "xyz"]
    save("torque_fcc10_dipole", d, keep)


CMC_TEMPS = (400.0, 900.0)
CMC_EQ, CMC_AV, CMC_EVERY = 2000, 20000, 10


def cmc_sc12():
    """Constrained Monte Carlo (montecarlo::cmc_step, src/montecarlo/cmc.cpp:
    282-490; sim:integrator=constrained-monte-carlo, angle moves) on SC 12^3
    periodic with the config-0 material, H = 0, constraint direction
    phi = 30, theta = 45 degrees: the reference's own chain at 400 K and
    900 K, 2,000 + 20,000 steps (N pair moves each), m sampled every 10
    steps; its constraint frame and move counters."""
    out = {}
    for T in CMC_TEMPS:
        inp = sc_input(12, T=T, H=0.0, integrator="constrained-monte-carlo",
                       extra="montecarlo:algorithm=angle\nsim:constraint-angle-phi=30\nsim:constraint-angle-theta=45\n")
        d = O.run_harness(inp, {"m.mat": SC_MAT}, ["--system", "--steps", CMC_EQ + CMC_AV, "--mag-every", CMC_EVERY,
                                                   "--mag-start", CMC_EQ], timeout=3600)
        tag = f"{int(T)}"
        out[f"m_trace_{tag}"] = d["mag_trace"].reshape(-1, 4)[:, :3].astype(np.float64)
        out[f"counters_{tag}"] = d["cmc_counters"]
        out["cmc_frame"] = d["cmc_frame"]
        for k in SYSTEM_KEYS:
            if k in d:
                out[k] = d[k]
    out["T"] = np.array(CMC_TEMPS)
    out["sweeps"] = np.array([CMC_EQ, CMC_AV, CMC_EVERY])
    np.savez_compressed(HERE / "cmc_sc12.npz", **out)
    print("cmc_sc12:", {T: out[f"counters_{int(T)}"] for T in CMC_TEMPS})


HYBRID_MAT = """material:num-materials=2
material[1]:material-name=A
material[1]:damping-constant=0.1
material[1]:exchange-matrix[1]=11.2e-21
material[1]:exchange-matrix[2]=8.0e-21
material[1]:atomic-spin-moment=1.72 !muB
material[1]:second-order-uniaxial-anisotropy-constant=6.69e-24
material[1]:uniaxial-anisotropy-direction=0,0,1
material[1]:constrained=true
material[1]:constraint-angle-phi=30
material[1]:constraint-angle-theta=45
material[1]:initial-spin-direction=0,0,1
material[2]:material-name=B
material[2]:damping-constant=0.1
material[2]:exchange-matrix[1]=8.0e-21
material[2]:exchange-matrix[2]=11.2e-21
material[2]:atomic-spin-moment=2.2 !muB
material[2]:second-order-uniaxial-anisotropy-constant=3.0e-24
material[2]:uniaxial-anisotropy-direction=0,0,1
material[2]:constrained=false
material[2]:initial-spin-direction=0,0,1
material[1]:host-alloy
material[1]:alloy-fraction[2]=0.5
"""


def cmc_hybrid_sc12():
    """Hybrid constrained Monte Carlo (montecarlo::cmc_mc_step,
    src/montecarlo/cmc_mc.cpp:291-490; sim:integrator=
    hybrid-constrained-monte-carlo): SC 12^3 periodic random A/B alloy
    (moments 1.72 and 2.2 mu_B), material A constrained along phi = 30,
    theta = 45 degrees, material B free; 500 K, 2,000 + 20,000 steps, the
    per-material magnetisation sampled every 10 steps; the reference's frames
    and counters."""
    inp = sc_input(12, T=500.0, H=0.0, integrator="hybrid-constrained-monte-carlo",
                   extra="montecarlo:algorithm=angle\n")
    d = O.run_harness(inp, {"m.mat": HYBRID_MAT}, ["--system", "--steps", CMC_EQ + CMC_AV, "--mag-every", CMC_EVERY,
                                                   "--mag-start", CMC_EQ], timeout=3600)
    keep = ["mat_trace", "cmc_frames", "cmc_counters"]
    d["sweeps"] = np.array([CMC_EQ, CMC_AV, CMC_EVERY])
    save("cmc_hybrid_sc12", d, keep + ["sweeps"])


MC50_EQ, MC50_AV = 5000, 10000


def autocorr_se(x: np.ndarray, c: float = 6.0):
    """Standard error of the mean of a correlated series from its integrated
    autocorrelation time, summed up to the first lag M >= c * tau (Sokal's
    self-consistent window).  Returns (se, tau in samples)."""
    x = np.asarray(x, dtype=np.float64) - np.mean(x)
    n = x.size
    var = float(x @ x) / n
    if var == 0.0:
        return 0.0, 0.0
    f = np.fft.rfft(x, 2 * n)
    rho = np.fft.irfft(f * np.conj(f))[:n] / (np.arange(n, 0, -1) * var)
    tau = 0.5
    for lag in range(1, n):
        tau += rho[lag]
        if lag >= c * tau:
            break
    return float(np.sqrt(2.0 * tau * var / n)), float(tau)


MC50_SEEDS = (None, 424242, 777001, 9051)


def _mc50_one(T, seed=None):
    extra = "montecarlo:algorithm=angle\n"
    if seed is not None:
        extra += f"sim:integrator-random-seed={seed}\n"
    inp = sc_input(50, T=T, H=0.0, integrator="monte-carlo", extra=extra)
    return O.run_harness(inp, {"m.mat": MC_MAT}, ["--system", "--steps", MC50_EQ + MC50_AV, "--mag-every", MC_EVERY,
                                                  "--mag-start", MC50_EQ], timeout=14400)


def mc_sc50_curie():
    """The Curie-sweep workload at its own size: the reference's sequential
    random-site Metropolis (montecarlo::mc_step, angle moves) on SC 50^3
    periodic (125,000 spins), config-0 material, H=0, spins start along z, 31
    temperatures 0..1500 K, 5,000 equilibration + 10,000 averaging sweeps,
    |m| sampled every 10 sweeps.  One reference process per temperature and
    chain (about 15 minutes each on one core); chains differ only in the
    reference's integrator seed (the first uses its default seed).
    MC50_CHAINS (default 2) sets the number of chains; chains already in the
    fixture with the same seed are kept, not re-run.  m_trace holds every
    chain's |m| series (chains, temperatures, samples); m_mean is the mean
    over chains.  A chain's standard error comes from its integrated
    autocorrelation time; with several chains these errors are checked
    against the spread of the chain means: kappa^2 = the mean over the
    finite temperatures of sum_c (m_c - m)^2 / se_c^2 / (chains - 1), and when
    kappa > 1 (the within-chain estimates too small: 10,000 sweeps hold only
    a few autocorrelation times near the transition) every error is scaled
    by kappa.  m_se is the standard error of m_mean."""
    from concurrent.futures import ThreadPoolExecutor
    import os
    workers = int(os.environ.get("MC50_WORKERS", os.cpu_count() or 4))
    nch = int(os.environ.get("MC50_CHAINS", 2))
    seeds = [(-1 if s is None else s) for s in MC50_SEEDS[:nch]]
    path = HERE / "mc_sc50_curie.npz"
    old = dict(np.load(path)) if path.exists() else {}
    have = {}
    if old:
        tr_old = old["m_trace"].reshape(-1, len(MC_TEMPS), old["m_trace"].shape[-1])
        acc_old = old["acceptance"].reshape(-1, len(MC_TEMPS))
        for k, s in enumerate(old.get("seeds", np.array([-1]))):
            have[int(s)] = (tr_old[k], acc_old[k])
    todo = [(T, s) for s in seeds if s not in have for T in MC_TEMPS]
    with ThreadPoolExecutor(workers) as ex:
        runs = list(ex.map(lambda a: _mc50_one(a[0], None if a[1] < 0 else a[1]), todo))
    for s in seeds:
        if s in have:
            continue
        mine = [d for (T, s2), d in zip(todo, runs) if s2 == s]
        tr = np.array([d["mag_trace"].reshape(-1, 4)[:, 3] for d in mine], dtype=np.float32)
        acc = np.array([1.0 - d["mc_counters"][1] / d["mc_counters"][0] for d in mine])
        have[s] = (tr, acc)
        if not old:
            old = {k: mine[0][k] for k in ("meta", "materials", "sim", "m_spin")}
    traces = np.stack([have[s][0] for s in seeds])          # (chains, T, samples)
    acc = np.stack([have[s][1] for s in seeds])
    means = traces.astype(np.float64).mean(2)
    ses = np.array([[autocorr_se(x)[0] for x in ch] for ch in traces])
    kappa = 1.0
    if len(seeds) > 1:
        live = np.all(ses > 0, axis=0)
        dev = (means[:, live] - means[:, live].mean(0)) ** 2 / ses[:, live] ** 2
        kappa = float(np.sqrt(dev.sum(0).mean() / (len(seeds) - 1)))
    scale = max(1.0, kappa)
    out = {k: old[k] for k in ("meta", "materials", "sim", "m_spin")}
    out.update(T=np.array(MC_TEMPS), m_mean=means.mean(0), m_se=scale * np.sqrt((ses ** 2).sum(0)) / len(seeds),
               chain_se=ses, kappa=np.array(kappa), acceptance=acc, m_trace=traces, seeds=np.array(seeds),
               L=np.array(50), sweeps=np.array([MC50_EQ, MC50_AV, MC_EVERY]))
    np.savez_compressed(path, **out)
    print("mc_sc50_curie:", np.round(out["m_mean"], 4), "kappa", round(kappa, 3))


def sc8_config():
    """The reference program's own configuration output (binary spin
    snapshots, src/config/atoms_spins.cpp) for the sc8_t0 input: the stock
    serial program with config:atoms every 5 output steps of 10 time steps,
    so snapshots at steps 10 and 60.  The spin data files and their meta files
    are kept as the reference wrote them."""
    import shutil
    import subprocess
    import tempfile
    from oracle.refinputs import SC_MAT, sc_input
    exe = HERE.parent.parent / "oracle" / "_ref" / "vampire-serial"
    d = Path(tempfile.mkdtemp(prefix="cfg_"))
    (d / "input").write_text(sc_input(8, T=0.0, extra="sim:total-time-steps=100\nsim:time-steps-increment=10\n"
                                                       "output:time-steps\noutput:magnetisation\nconfig:atoms\n"
                                                       "config:atoms-output-rate=5\nconfig:output-format=binary\n"))
    (d / "m.mat").write_text(SC_MAT)
    subprocess.run([str(exe)], cwd=d, check=True, capture_output=True, timeout=600)
    out = HERE / "sc8_config"
    out.mkdir(exist_ok=True)
    for f in ("spins-00000000.data", "spins-00000000.meta", "spins-00000001.data", "spins-00000001.meta"):
        shutil.copy(d / f, out / f)
    print("sc8_config:", sorted(p.name for p in out.iterdir()))


ALL = [sc20_t0, sc8_t0, sc10_t300, sc6_open_t300, fcc4_dmi_t300, fcc4_dmi_t0, single_spin_applied, mc_sc16_curie,
       mc_sc50_curie, tet_bond_exchange, sc6_vec, torque_fixtures, cmc_sc12, cmc_hybrid_sc12,
       fcc10_dipole_tensor, fcc10_dipole_macrocell, sc6_aniso_ho, fcc4_neel_rot, sc6_derived_t600, sc8_midpoint, sc6_biquadratic,
       sc8_config]

if __name__ == "__main__":
    names = sys.argv[1:]
    for f in ALL:
        if not names or f.__name__ in names:
            f()
