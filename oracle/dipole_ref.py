"""NumPy restatement of the reference macrocell dipole field (dense, small
systems).  TEST INFRASTRUCTURE ONLY.

Follows cells::mag (src/cells/mag.cpp:35-77), the tensor solver's inter and
intra tensors (src/dipole/inter.cpp:40-150, src/dipole/intra.cpp:40-140),
the macrocell solver (src/dipole/macrocell.cpp:175-225) and
dipole::internal::update_field (src/dipole/update.cpp:37-105).
"""
from __future__ import annotations

import numpy as np

MU_B = 9.27400915e-24


def cell_moments(spins, mu_s_SI_per_atom, atom_cell, nc, magnetic=None):
    m = np.zeros((3, nc))
    w = mu_s_SI_per_atom if magnetic is None else np.where(magnetic, mu_s_SI_per_atom, 0.0)
    for q in range(3):
        np.add.at(m[q], atom_cell, spins[q] * w)
    return m


def tensors(cell_pos, natoms, size, cutoff, solver, coords=None, atom_cell=None):
    """Dense (6, nc, nc) interaction tensors xx, xy, xz, yy, yz, zz."""
    nc = natoms.size
    T = np.zeros((6, nc, nc))
    P = cell_pos.reshape(nc, 4)[:, :3]
    members = None
    if solver == "tensor":
        members = [np.nonzero(atom_cell == c)[0] for c in range(nc)]
    for i in range(nc):
        if natoms[i] <= 0:
            continue
        for j in range(nc):
            if natoms[j] <= 0:
                continue
            if i != j:
                r = P[j] - P[i]
                rij = 1.0 / np.sqrt(r @ r)
                if solver == "macrocell" or (1.0 / rij) / size > cutoff:
                    e = r * rij
                    r3 = rij ** 3
                    T[:, i, j] = [(3 * e[0] * e[0] - 1) * r3, 3 * e[0] * e[1] * r3, 3 * e[0] * e[2] * r3,
                                  (3 * e[1] * e[1] - 1) * r3, 3 * e[1] * e[2] * r3, (3 * e[2] * e[2] - 1) * r3]
                    continue
            elif solver == "macrocell":
                continue
            a = coords[:, members[i]].T
            b = coords[:, members[j]].T
            d = b[None, :, :] - a[:, None, :]
            r2 = (d * d).sum(-1)
            ok = r2 > 0
            rij = np.where(ok, 1.0 / np.sqrt(np.where(ok, r2, 1.0)), 0.0)
            e = d * rij[..., None]
            r3 = rij ** 3
            comps = [(3 * e[..., 0] ** 2 - 1), 3 * e[..., 0] * e[..., 1], 3 * e[..., 0] * e[..., 2],
                     (3 * e[..., 1] ** 2 - 1), 3 * e[..., 1] * e[..., 2], (3 * e[..., 2] ** 2 - 1)]
            for k in range(6):
                T[k, i, j] = (np.where(ok, comps[k] * r3, 0.0)).sum() / (float(natoms[i]) * float(natoms[j]))
    return T


def cell_fields(mag, T, natoms, volume):
    """(B, mu0 Hd), each (3, nc), in Tesla (update.cpp:56-99)."""
    m = mag / MU_B
    xx, xy, xz, yy, yz, zz = T
    f = np.stack([xx @ m[0] + xy @ m[1] + xz @ m[2],
                  xy @ m[0] + yy @ m[1] + yz @ m[2],
                  xz @ m[0] + yz @ m[1] + zz @ m[2]])
    has = natoms > 0
    self_ = np.where(has, 8.0 * np.pi / (3.0 * np.where(has, volume, 1.0)), 0.0)
    B = np.where(has, f * 9.27400915e-01, 0.0)
    H = np.where(has, (f - 0.5 * self_ * m) * 9.27400915e-01, 0.0)
    return B, H
