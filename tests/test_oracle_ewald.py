"""The oracle's Ewald electrostatics on the rock-salt crystal, whose Madelung
constant is known (no GPU): E = E_real + E_recip + E_self per ion pair equals
-1.747565 K / r0."""
import numpy as np

from pygcmc_b200 import values as V
from pygcmc_b200.system import System

K = 1388.431112
MADELUNG_NACL = 1.7475645946


def ionic_system(ncell=3, a=5.64):
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    pos, q = [], []
    for i in range(ncell):
        for j in range(ncell):
            for k in range(ncell):
                for b in base:
                    pos.append((np.array([i, j, k]) + b) * a)
                    q.append(1.0)
                    pos.append((np.array([i, j, k]) + b + [0.5, 0, 0]) * a)
                    q.append(-1.0)
    pos, q = np.array(pos), np.array(q)
    n = len(pos)
    L = ncell * a
    info = np.zeros(1, dtype=V.Info_dtype)
    info[0]["cryst"] = [L, L, L]
    info[0]["cutoff"] = L / 2 - 0.01
    info[0]["fragTypeNum"] = 1
    info[0]["totalResNum"] = n
    info[0]["totalAtomNum"] = n
    frag = np.zeros(1, dtype=V.AtomArray_dtype)
    frag[0]["startRes"] = n
    res = np.zeros(n, dtype=V.Residue_dtype)
    res["atomStart"] = np.arange(n)
    res["atomNum"] = 1
    res["position"] = pos
    atoms = np.zeros(n, dtype=V.Atom_dtype)
    atoms["position"] = pos
    atoms["charge"] = q
    return System(info, frag, res, atoms, np.zeros(3, np.float32), np.zeros(2, np.float32), np.zeros(0, np.int32)), pos, q, L


def test_ewald_reproduces_the_madelung_constant(oracle_lib):
    from scipy.special import erfc
    s, pos, q, L = ionic_system()
    alpha = 0.45
    phi = oracle_lib.ewald_potential(s, alpha, pos)
    e_rec = 0.5 * np.dot(q, phi)
    rc = 7.0  # real-space cutoff: erfc(0.45 * 7) ~ 1e-5 relative
    e_real = 0.0
    shifts = np.array([[i, j, k] for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)]) * L
    for i in range(len(pos)):
        d = pos[None, :, :] + shifts[:, None, :] - pos[i]
        r = np.linalg.norm(d, axis=2)
        m = (r > 1e-9) & (r < rc)
        e_real += 0.5 * K * q[i] * np.sum((q[None, :] * erfc(alpha * r) / np.where(m, r, 1.0))[m])
    e_self = -K * alpha / np.sqrt(np.pi) * np.sum(q * q)
    per_pair = (e_real + e_rec + e_self) / (len(q) / 2)
    r0 = 5.64 / 2
    assert abs(per_pair + MADELUNG_NACL * K / r0) < 2e-4 * MADELUNG_NACL * K / r0, (per_pair, -MADELUNG_NACL * K / r0)
