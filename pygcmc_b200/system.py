"""Builders of the seven GCMC state arrays, and seeded synthetic systems.

The builders restate pyGCMC's input assembly for the hot path:

* :func:`cavity_grid`      -- ``GCMCDataset.get_grid``   (gcmc/python/dataset.py:21-139)
* :func:`move_array`       -- ``GCMCDataset.get_move``   (gcmc/python/dataset.py:141-171)
* :func:`fix_groups`       -- ``GCMCDataset.set_fixCut`` (gcmc/python/dataset.py:175-188)
* :func:`lj_pair_table`    -- ``GCMCSimulation.get_simulation`` type/LJ tables
  (gcmc/python/simulation.py:56-75)
* :func:`assemble`         -- ``GCMCDataset.update_data`` (gcmc/python/dataset.py:190-373)

Differences from the reference are deliberate and few: the cavity-grid voxels
are listed in lexicographic (x, y, z) order instead of Python ``set`` order,
and unused slots are zero-filled instead of left uninitialised.

The synthetic systems stand in for the benchmark inputs (no public dataset is
involved): a TIP3P water box, a random-walk "protein" with eight generic rigid
fragments, and batches of such systems of uneven size.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import random
from typing import List, Optional, Sequence

import numpy as np

from . import values as V
from ._native import check, lib, ptr


# ---------------------------------------------------------------------------
# state container
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class System:
    """The seven arrays passed to ``runGCMC`` plus descriptive metadata."""
    SimInfo: np.ndarray
    fragmentInfo: np.ndarray
    residueInfo: np.ndarray
    atomInfo: np.ndarray
    grid: np.ndarray
    ff: np.ndarray
    moveArray: np.ndarray
    meta: dict = dataclasses.field(default_factory=dict)
    # the cavity grid as a gcmc_grid_bits record (uint8: 48-byte header + voxel words), or None
    grid_bits: Optional[np.ndarray] = None

    def arrays(self):
        return (self.SimInfo, self.fragmentInfo, self.residueInfo, self.atomInfo, self.grid, self.ff,
                self.moveArray)

    def arrays_for(self, options=None):
        """The seven arrays a run entry point takes under ``options``: with
        ``options.grid_bits`` set, the ``grid`` slot carries the voxel bit set
        (:attr:`grid_bits`) instead of the float list."""
        a = self.arrays()
        if options is not None and getattr(options, "grid_bits", 0):
            if self.grid_bits is None:
                raise ValueError("options.grid_bits is set but this System carries no grid_bits record")
            a = a[:4] + (self.grid_bits,) + a[5:]
        return a

    def copy(self) -> "System":
        return System(*(a.copy() for a in self.arrays()), meta=dict(self.meta),
                      grid_bits=None if self.grid_bits is None else self.grid_bits.copy())

    def pinned(self) -> "System":
        """A copy whose arrays live in page-locked host memory (needs torch with
        CUDA).  The drop-in calls copy page-locked arrays to and from the GPU
        directly instead of through the driver's staging buffers."""
        import torch
        keep, arrs = [], []
        extra = () if self.grid_bits is None else (self.grid_bits,)
        for a in self.arrays() + extra:
            buf = torch.empty(max(1, a.nbytes), dtype=torch.uint8, pin_memory=True)
            v = buf.numpy()[:a.nbytes].view(a.dtype).reshape(a.shape)
            v[...] = a
            keep.append(buf)
            arrs.append(v)
        out = System(*arrs[:7], meta=dict(self.meta), grid_bits=arrs[7] if extra else None)
        out._page_locked = keep  # the buffers the arrays view
        return out

    def moved_bytes(self) -> int:
        """Bytes a drop-in call copies back to the host: the fragment types'
        counts, the fragment residues' centres and the fragment slots' atoms
        (position + charge, type)."""
        g0 = int(self.fragmentInfo[0]["startRes"])
        res = self.residueInfo[g0:]
        if len(res) == 0:
            return 4 * len(self.fragmentInfo)
        lo = int(res["atomStart"].min())
        hi = int((res["atomStart"] + res["atomNum"]).max())
        return 4 * len(self.fragmentInfo) + 16 * len(res) + 20 * max(0, hi - lo)

    @property
    def info(self):
        return self.SimInfo[0]

    def n_fixed_atoms(self) -> int:
        s0 = int(self.fragmentInfo[0]["startRes"])
        return int(self.residueInfo[s0]["atomStart"]) if s0 < len(self.residueInfo) else 0


# ---------------------------------------------------------------------------
# reference input builders
# ---------------------------------------------------------------------------
def cavity_grid(xyz: np.ndarray, cryst: Sequence[float], grid_dx: float = 1.0, cavity_bias: bool = True):
    """Box origin, insertion base points and cavity factor (dataset.py:21-139), in C++
    (``gcmc_cavity_grid``).

    The box is centred on the bounding box of all atoms; voxels of edge
    ``grid_dx`` that contain no atom are the insertion base points (their
    lower corners) and ``cavity_factor = empty / all``.  Without cavity bias
    every voxel of a 1 A grid is used and the factor is 1.
    """
    xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
    cr = np.ascontiguousarray([float(c) for c in cryst], dtype=np.float64)
    start = np.zeros(3, np.float64)
    n = ctypes.c_int64(0)
    factor = ctypes.c_double(0.0)
    L = lib()
    st = L.gcmc_cavity_grid(len(xyz), ptr(xyz), ptr(cr), float(grid_dx), int(bool(cavity_bias)), ptr(start), None, 0,
                            ctypes.byref(n), ctypes.byref(factor))
    if st == 2 and cavity_bias:
        raise ValueError("cavity_bias_factor is too small (< 0.05); decrease the grid spacing")
    check(st, "gcmc_cavity_grid")
    pts = np.empty(3 * n.value, dtype=np.float32)
    check(L.gcmc_cavity_grid(len(xyz), ptr(xyz), ptr(cr), float(grid_dx), int(bool(cavity_bias)), ptr(start),
                             ptr(pts), n.value, ctypes.byref(n), ctypes.byref(factor)), "gcmc_cavity_grid")
    dx = float(grid_dx) if cavity_bias else 1.0
    return [float(v) for v in start], pts, factor.value, dx


GRID_BITS_HEADER = 48  # sizeof(gcmc_grid_bits)


def cavity_bits(xyz: np.ndarray, cryst: Sequence[float], grid_dx: float = 1.0, cavity_bias: bool = True):
    """The grid of :func:`cavity_grid` as a ``gcmc_grid_bits`` record
    (``gcmc_cavity_bits``): a uint8 array holding the 48-byte header (voxel
    (0, 0, 0) corner, edge, voxels per axis) and one bit per voxel, set for the
    insertion base points.  Runs with ``Options.grid_bits = 1`` take it in
    place of the float list: the same points in the same order, 1 bit per voxel
    instead of 12 bytes per point on the way to the device."""
    xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
    cr = np.ascontiguousarray([float(c) for c in cryst], dtype=np.float64)
    nw, npts = ctypes.c_int64(0), ctypes.c_int64(0)
    hdr = np.zeros(GRID_BITS_HEADER, np.uint8)
    L = lib()
    st = L.gcmc_cavity_bits(len(xyz), ptr(xyz), ptr(cr), float(grid_dx), int(bool(cavity_bias)), ptr(hdr), None, 0,
                            ctypes.byref(nw), ctypes.byref(npts))
    if st == 2 and cavity_bias:
        raise ValueError("cavity_bias_factor is too small (< 0.05); decrease the grid spacing")
    check(st, "gcmc_cavity_bits")
    out = np.zeros(GRID_BITS_HEADER + 4 * nw.value, np.uint8)
    words = out[GRID_BITS_HEADER:].view(np.uint32)
    check(L.gcmc_cavity_bits(len(xyz), ptr(xyz), ptr(cr), float(grid_dx), int(bool(cavity_bias)), ptr(out),
                             ptr(words), nw.value, ctypes.byref(nw), ctypes.byref(npts)), "gcmc_cavity_bits")
    return out


def move_array(nsteps: int, names: Sequence[str], mctime: Sequence[float],
               attempt_prob_frag=(0.3, 0.3, 0.2, 0.2), attempt_prob_water=(0.25, 0.25, 0.25, 0.25),
               rng: Optional[random.Random] = None) -> np.ndarray:
    """``moveArray[i] = fragType*4 + move`` (dataset.py:141-171), Python ``random`` draws."""
    rng = rng or random.Random()
    frag = rng.choices(range(len(names)), weights=mctime, k=nsteps)
    out = np.empty(nsteps, dtype=np.int32)
    for i, f in enumerate(frag):
        w = attempt_prob_water if names[f] == "SOL" else attempt_prob_frag
        out[i] = f * 4 + rng.choices(range(len(w)), weights=w, k=1)[0]
    return out


def move_array_np(nsteps: int, names: Sequence[str], mctime: Sequence[float],
                  attempt_prob_frag=(0.3, 0.3, 0.2, 0.2), attempt_prob_water=(0.25, 0.25, 0.25, 0.25),
                  seed: int = 0) -> np.ndarray:
    """Same law as :func:`move_array`, drawn with numpy (fast for 1e6+ steps)."""
    g = np.random.default_rng(seed)
    p = np.asarray(mctime, dtype=np.float64)
    frag = g.choice(len(names), size=nsteps, p=p / p.sum())
    pw = np.asarray(attempt_prob_water, dtype=np.float64)
    pf = np.asarray(attempt_prob_frag, dtype=np.float64)
    is_sol = np.array([n == "SOL" for n in names])[frag]
    mv = np.where(is_sol, g.choice(4, size=nsteps, p=pw / pw.sum()), g.choice(4, size=nsteps, p=pf / pf.sum()))
    return (frag * 4 + mv).astype(np.int32)


def fix_groups(xyz: np.ndarray, fix_cutoff: float = 6.0) -> np.ndarray:
    """Group id per fixed atom (dataset.py:175-188), in C++ (``gcmc_fix_groups``): a
    new group starts when an atom lies more than ``fix_cutoff`` from the current
    group's first atom."""
    xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
    out = np.empty(len(xyz), dtype=np.int32)
    if len(xyz) and lib().gcmc_fix_groups(len(xyz), ptr(xyz), float(fix_cutoff), ptr(out)) < 0:
        raise ValueError("gcmc_fix_groups")
    return out.astype(np.int64)


def lj_pair_table(frag_types: Sequence[str], env_types: Sequence[str], nb: dict, nbfix: Optional[dict] = None):
    """Type tables and the LJ pair table (simulation.py:56-75).

    ``nb[type] = (sigma_nm, eps_kJ)``.  Rows are the fragment types in order of
    appearance, columns all types (fragment types first); pair parameters come
    from ``nbfix`` when present, else Lorentz-Berthelot combining.
    Returns ``(atomtypes1, atomtypes2, ff)`` with ``ff`` float32 of length
    ``2*len(atomtypes1)*len(atomtypes2)``.
    """
    nbfix = nbfix or {}
    t1, t2 = [], []
    for t in frag_types:
        if t not in t2:
            t1.append(t)
            t2.append(t)
    for t in env_types:
        if t not in t2:
            t2.append(t)
    ff = np.empty(2 * len(t1) * len(t2), dtype=np.float32)
    k = 0
    for a in t1:
        for b in t2:
            if (a, b) in nbfix:
                s, e = nbfix[(a, b)]
            elif (b, a) in nbfix:
                s, e = nbfix[(b, a)]
            else:
                s = (nb[a][0] + nb[b][0]) / 2
                e = np.sqrt(nb[a][1] * nb[b][1])
            ff[2 * k] = s
            ff[2 * k + 1] = e
            k += 1
    return t1, t2, ff


def group_centres(xyz: np.ndarray, starts: np.ndarray, counts: np.ndarray) -> np.ndarray:
    """Unweighted group centres with the reference's arithmetic (dataset.py:248-300
    under its numpy<2 dependency), in C++ (``gcmc_group_centres``): each coordinate
    is added in float64 to a float32 running sum that is rounded back to float32,
    then divided by the count in float64 and stored as float32."""
    xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
    starts = np.ascontiguousarray(starts, dtype=np.int64)
    counts = np.ascontiguousarray(counts, dtype=np.int32)
    out = np.zeros((len(starts), 3), dtype=np.float32)
    check(lib().gcmc_group_centres(len(starts), ptr(xyz), ptr(starts), ptr(counts), ptr(out)), "gcmc_group_centres")
    return out


def charmm_to_nb(eps_kcal: float, rmin_half: float):
    """CHARMM (epsilon [kcal/mol], Rmin/2 [A]) -> (sigma [nm], epsilon [kJ/mol])."""
    return (2.0 * rmin_half / 2.0 ** (1.0 / 6.0) / 10.0, V.KCAL_TO_KJ * eps_kcal)


def assemble(*, names: Sequence[str], templates: Sequence[dict], initial: Sequence[Sequence[np.ndarray]],
             fixed_xyz: np.ndarray, fixed_q: np.ndarray, fixed_type: np.ndarray, fixed_group: np.ndarray,
             muex, conc, conf_bias, mctime, cryst, cutoff: float, grid_dx: float, start, grid: np.ndarray,
             cavity_factor: float, ff: np.ndarray, n_frag_types_ff: int, n_types_ff: int, moves: np.ndarray,
             seed: int, show_info: int = 0, pme: int = 0) -> System:
    """``update_data`` (dataset.py:190-373): fragment table, slot layout, atoms, SimInfo.

    ``templates[i]`` = ``{"xyz": (n,3), "q": (n,), "type": (n,)}`` (type = column
    index of ff); ``initial[i]`` = list of (n,3) site arrays already in the box.
    Group centres follow the reference's arithmetic (see :func:`group_centres`).
    """
    nt = len(names)
    volume = float(cryst[0]) * float(cryst[1]) * float(cryst[2])
    n_ins = np.bincount(moves[(moves % 4) == 0] // 4, minlength=nt) if len(moves) else np.zeros(nt, int)
    frag = np.zeros(nt, dtype=V.AtomArray_dtype)
    for i in range(nt):
        t = templates[i]
        xyz = np.asarray(t["xyz"], dtype=np.float64)
        xyz = xyz - np.cumsum(xyz, axis=0)[-1] / len(xyz)  # sequential sum, as dataset.py:219-222
        frag[i]["name"] = names[i].ljust(4)[:4].encode()
        frag[i]["muex"] = muex[i]
        frag[i]["conc"] = conc[i]
        frag[i]["confBias"] = conf_bias[i]
        frag[i]["mcTime"] = mctime[i]
        frag[i]["totalNum"] = len(initial[i])
        m1 = conc[i] * volume * V.MOLES_TO_MOLECULES * 2 + n_ins[i]
        m2 = len(initial[i]) + n_ins[i]
        frag[i]["maxNum"] = int(max(m1, m2))
        frag[i]["num_atoms"] = len(xyz)
        frag[i]["atoms"]["position"][: len(xyz)] = xyz
        frag[i]["atoms"]["charge"][: len(xyz)] = t["q"]
        frag[i]["atoms"]["type"][: len(xyz)] = t["type"]
    nfix = len(fixed_xyz)
    fixed_group = np.ascontiguousarray(fixed_group, dtype=np.int32)
    ngroups_fixed = int(np.count_nonzero(np.diff(fixed_group))) + 1 if nfix else 0
    total_res = ngroups_fixed + int(frag["maxNum"].sum())
    total_atoms = nfix + int((frag["maxNum"].astype(np.int64) * frag["num_atoms"]).sum())
    res = np.zeros(total_res, dtype=V.Residue_dtype)
    atoms = np.zeros(total_atoms, dtype=V.Atom_dtype)
    # residue / atom arrays in C++ (gcmc_fill_layout)
    fx = np.ascontiguousarray(np.asarray(fixed_xyz, dtype=np.float64).reshape(-1, 3))
    fq = np.ascontiguousarray(fixed_q, dtype=np.float64)
    ft = np.ascontiguousarray(fixed_type, dtype=np.int32)
    tq = np.ascontiguousarray(np.concatenate([np.asarray(t["q"], np.float32) for t in templates]), dtype=np.float32)
    tt = np.ascontiguousarray(np.concatenate([np.asarray(t["type"], np.int32) for t in templates]), dtype=np.int32)
    ninit = np.ascontiguousarray([len(c) for c in initial], dtype=np.int32)
    parts = [np.asarray(p, dtype=np.float64).reshape(-1, 3) for c in initial for p in c]
    ixyz = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros((0, 3)), dtype=np.float64)
    start_res = np.zeros(nt, dtype=np.int32)
    check(lib().gcmc_fill_layout(nfix, ptr(fx), ptr(fq), ptr(ft), ptr(fixed_group), nt,
                                 ptr(np.ascontiguousarray(frag["maxNum"], np.int32)),
                                 ptr(np.ascontiguousarray(frag["num_atoms"], np.int32)), ptr(tq), ptr(tt), ptr(ninit),
                                 ptr(ixyz), total_res, total_atoms, ptr(res), ptr(atoms), ptr(start_res)),
          "gcmc_fill_layout")
    frag["startRes"] = start_res
    info = np.zeros(1, dtype=V.Info_dtype)
    info[0]["ffXNum"] = n_frag_types_ff
    info[0]["ffYNum"] = n_types_ff
    info[0]["mcsteps"] = len(moves)
    info[0]["cutoff"] = cutoff
    info[0]["grid_dx"] = grid_dx
    info[0]["startxyz"] = start
    info[0]["cryst"] = cryst
    info[0]["cavityFactor"] = cavity_factor
    info[0]["fragTypeNum"] = nt
    info[0]["totalGridNum"] = len(grid) // 3
    info[0]["totalResNum"] = total_res
    info[0]["totalAtomNum"] = total_atoms
    info[0]["showInfo"] = show_info
    info[0]["PME"] = pme
    info[0]["seed"] = seed & 0xFFFFFFFF
    return System(info, frag, res, atoms, np.ascontiguousarray(grid, dtype=np.float32),
                  np.ascontiguousarray(ff, dtype=np.float32), np.ascontiguousarray(moves, dtype=np.int32),
                  meta={"names": list(names)})


# ---------------------------------------------------------------------------
# geometry helpers for the synthetic systems
# ---------------------------------------------------------------------------
def random_rotation(g: np.random.Generator) -> np.ndarray:
    """Uniform random rotation matrix (quaternion of four normals)."""
    q = g.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def tip3p_template():
    """TIP3P water: O-H 0.9572 A, H-O-H 104.52 degrees, O at the origin."""
    half = math.radians(104.52) / 2
    b = 0.9572
    xyz = np.array([[0.0, 0.0, 0.0], [b * math.sin(half), b * math.cos(half), 0.0],
                    [-b * math.sin(half), b * math.cos(half), 0.0]])
    return xyz


def lattice_template(g: np.random.Generator, n: int, kind: str, bond: float = 1.4) -> np.ndarray:
    """n sites on a honeycomb (planar) or diamond (tetrahedral) lattice walk with bond length `bond`."""
    if kind == "planar":
        dirs_a = np.array([[1.0, 0.0, 0.0], [-0.5, math.sqrt(3) / 2, 0.0], [-0.5, -math.sqrt(3) / 2, 0.0]])
        dirs = [dirs_a, -dirs_a]
    else:
        t = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=np.float64) / math.sqrt(3)
        dirs = [t, -t]
    pts = [np.zeros(3)]
    parity = [0]
    keys = {tuple(np.round(pts[0], 3))}
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > 10000:
            raise RuntimeError("template walk stuck")
        base = g.integers(len(pts))
        d = dirs[parity[base]][g.integers(len(dirs[0]))]
        p = pts[base] + bond * d
        key = tuple(np.round(p, 3))
        if key in keys:
            continue
        keys.add(key)
        pts.append(p)
        parity.append(1 - parity[base])
    xyz = np.array(pts)
    return xyz - xyz.mean(axis=0)


def _min_image(d, L):
    return d - L * np.round(d / L)


def _place_rigid(g, template, count, L, start, existing, min_dist, max_tries=20000):
    """Random non-clashing copies of a template inside the periodic box."""
    out = []
    pool = [existing] if len(existing) else []
    Lv = np.asarray(L, dtype=np.float64)
    for _ in range(count):
        for _t in range(max_tries):
            c = np.asarray(start) + g.random(3) * Lv
            p = template @ random_rotation(g).T + c
            ok = True
            for blk in pool:
                d = _min_image(blk[:, None, :] - p[None, :, :], Lv)
                if (np.einsum("ijk,ijk->ij", d, d) < min_dist * min_dist).any():
                    ok = False
                    break
            if ok:
                out.append(p)
                pool.append(p)
                break
        else:
            raise RuntimeError("could not place fragment copy")
    return out


# ---------------------------------------------------------------------------
# synthetic systems
# ---------------------------------------------------------------------------
def water_box(n_water: int = 800, box: float = 30.0, seed: int = 1, mcsteps: int = 100_000,
              conf_bias: int = 1000, muex: float = -5.8, conc: float = 55.0, cutoff: float = 12.0,
              grid_dx: float = 1.0, moves: Optional[np.ndarray] = None) -> System:
    """TIP3P water box (no fixed atoms): O uniform with O-O >= 2.6 A, random orientations."""
    g = np.random.default_rng(seed)
    tpl = tip3p_template()
    L = np.array([box, box, box])
    ox = []
    while len(ox) < n_water:
        p = g.random(3) * L
        if ox:
            d = _min_image(np.asarray(ox) - p, L)
            if (np.einsum("ij,ij->i", d, d) < 2.6 ** 2).any():
                continue
        ox.append(p)
    waters = [tpl @ random_rotation(g).T + o for o in ox]
    xyz_all = np.concatenate(waters)
    nb = {"OT": charmm_to_nb(0.1521, 1.7682), "HT": charmm_to_nb(0.046, 0.2245)}
    t1, t2, ff = lj_pair_table(["OT", "HT", "HT"], [], nb)
    start, grid, cav, dx = cavity_grid(xyz_all, L, grid_dx)
    if moves is None:
        moves = move_array_np(mcsteps, ["SOL"], [1.0], seed=seed)
    tpl_c = {"xyz": tpl, "q": np.array([-0.834, 0.417, 0.417]), "type": np.array([0, 1, 1])}
    s = assemble(names=["SOL"], templates=[tpl_c], initial=[waters], fixed_xyz=np.zeros((0, 3)),
                 fixed_q=np.zeros(0), fixed_type=np.zeros(0, int), fixed_group=np.zeros(0, int),
                 muex=[muex], conc=[conc], conf_bias=[conf_bias], mctime=[1.0], cryst=L, cutoff=cutoff,
                 grid_dx=dx, start=start, grid=grid, cavity_factor=cav, ff=ff, n_frag_types_ff=len(t1),
                 n_types_ff=len(t2), moves=moves, seed=seed)
    s.grid_bits = cavity_bits(xyz_all, L, grid_dx)
    return s


def protein_system(seed: int = 1, n_atoms: int = 6000, box: float = 64.0, radius: float = 24.0,
                   n_frag: int = 8, n_types: int = 24, mcsteps: int = 1_000_000, conf_bias: int = 1000,
                   conc: float = 0.25, cutoff: float = 12.0, grid_dx: float = 1.0, excl: float = 1.6,
                   n_initial: Optional[int] = None, muex_shift: float = 0.0,
                   moves: Optional[np.ndarray] = None) -> System:
    """Random-walk protein in a periodic box with generic rigid fragments.

    Fixed atoms: a confined self-avoiding walk (1.5 A steps) in a sphere at the
    box centre; ``excl`` is the non-bonded exclusion distance (6000 atoms in a
    24 A sphere is 0.10 atoms/A^3, above close packing for 3 A spheres, so the
    default uses 1.6 A).  24 LJ types with epsilon ~ U[0.02, 0.20] kcal/mol and
    Rmin/2 ~ U[1.0, 2.2] A, charges ~ N(0, 0.35) shifted to zero net.
    Fragments: 4-12 sites on a 1.4 A planar or tetrahedral lattice, charges
    ~ N(0, 0.3) shifted to a total of 0 or +-1, types from the same 24,
    muex ~ U[-5, -1] (+ muex_shift).  Each type starts with
    round(conc * V * 6.023e-4) copies placed without clashes (>= 2 A).
    """
    g = np.random.default_rng(seed)
    L = np.array([box, box, box], dtype=np.float64)
    centre = (L / 2).astype(np.float32)
    xyz = np.empty((n_atoms, 3), dtype=np.float32)
    nbreak = __import__("ctypes").c_int(0)
    rc = lib().gcmc_synth_chain_sphere(n_atoms, ptr(centre), radius, 1.5, excl, int(seed) * 7919 + 17, ptr(xyz),
                                       __import__("ctypes").byref(nbreak))
    if rc != 0:
        raise RuntimeError("chain generation failed (sphere too small for the exclusion distance)")
    tnames = [f"T{i:02d}" for i in range(n_types)]
    eps = g.uniform(0.02, 0.20, n_types)
    rmin2 = g.uniform(1.0, 2.2, n_types)
    nb = {tnames[i]: charmm_to_nb(eps[i], rmin2[i]) for i in range(n_types)}
    q = g.normal(0.0, 0.35, n_atoms)
    q -= q.mean()
    ptype = g.integers(n_types, size=n_atoms)
    names, templates_raw = [], []
    for f in range(n_frag):
        ns = int(g.integers(4, 13))
        kind = "planar" if g.random() < 0.5 else "tetrahedral"
        txyz = lattice_template(g, ns, kind)
        tq = g.normal(0.0, 0.3, ns)
        tq += (int(g.integers(-1, 2)) - tq.sum()) / ns
        tt = g.integers(n_types, size=ns)
        names.append(f"FR{f:02d}")
        templates_raw.append((txyz, tq, tt))
    frag_type_names = [tnames[t] for (_, _, tt) in templates_raw for t in tt]
    t1, t2, ff = lj_pair_table(frag_type_names, [tnames[t] for t in ptype], nb)
    col = {t: i for i, t in enumerate(t2)}
    templates = [{"xyz": txyz, "q": tq, "type": np.array([col[tnames[t]] for t in tt])}
                 for (txyz, tq, tt) in templates_raw]
    fixed_type = np.array([col[tnames[t]] for t in ptype])
    muex = (g.uniform(-5.0, -1.0, n_frag) + muex_shift).tolist()
    if n_initial is None:
        n_initial = int(round(conc * float(np.prod(L)) * V.MOLES_TO_MOLECULES))
    initial = []
    existing = np.ascontiguousarray(xyz, dtype=np.float32)
    lo = np.zeros(3, np.float32)
    Lf = L.astype(np.float32)
    for f in range(n_frag):
        tx = np.ascontiguousarray(templates[f]["xyz"] - templates[f]["xyz"].mean(axis=0), dtype=np.float32)
        ns = len(tx)
        out = np.zeros((n_initial, ns, 3), np.float32)
        if n_initial:
            rc = lib().gcmc_synth_place(len(existing), ptr(existing), ptr(lo), ptr(Lf), ptr(tx), ns, n_initial, 2.0,
                                        int(seed) * 104729 + 31 * f + 7, ptr(out))
            if rc != 0:
                raise RuntimeError("could not place the initial fragment copies")
            existing = np.ascontiguousarray(np.concatenate([existing, out.reshape(-1, 3)]))
        initial.append([out[c].astype(np.float64) for c in range(n_initial)])
    all_xyz = existing.astype(np.float64)
    start, grid, cav, dx = cavity_grid(all_xyz, L, grid_dx)
    groups = fix_groups(xyz, 6.0)
    if moves is None:
        moves = move_array_np(mcsteps, names, [1.0] * n_frag, seed=seed + 1)
    s = assemble(names=names, templates=templates, initial=initial, fixed_xyz=xyz, fixed_q=q,
                 fixed_type=fixed_type, fixed_group=groups, muex=muex, conc=[conc] * n_frag,
                 conf_bias=[conf_bias] * n_frag, mctime=[1.0] * n_frag, cryst=L, cutoff=cutoff, grid_dx=dx,
                 start=start, grid=grid, cavity_factor=cav, ff=ff, n_frag_types_ff=len(t1), n_types_ff=len(t2),
                 moves=moves, seed=seed)
    s.grid_bits = cavity_bits(all_xyz, L, grid_dx)
    s.meta.update({"chain_breaks": int(nbreak.value), "n_fixed": n_atoms, "box": box,
                   # per-type CHARMM parameters in the ff column order (t2); rows are t2[:ffX]
                   "lj_types": {"names": list(t2), "eps_kcal": np.array([eps[tnames.index(n)] for n in t2]),
                                "rmin_half": np.array([rmin2[tnames.index(n)] for n in t2])}})
    return s


def replica_batch(n_rep: int = 64, seed: int = 1, atoms_range=(2000, 40000), mcsteps: int = 100_000,
                  conf_bias: int = 1000, density: float = 6000 / 64.0 ** 3) -> List[System]:
    """Replicas of uneven size: protein atoms log-uniform in ``atoms_range``, box
    edge scaled to keep the protein density (clamped to [40, 100] A), replica i's
    muex shifted by -8 + 8 i / (n_rep - 1)."""
    g = np.random.default_rng(seed)
    out = []
    for i in range(n_rep):
        n = int(round(math.exp(g.uniform(math.log(atoms_range[0]), math.log(atoms_range[1])))))
        box = float(np.clip((n / density) ** (1.0 / 3.0), 40.0, 100.0))
        radius = 24.0 * (n / 6000.0) ** (1.0 / 3.0)
        radius = min(radius, box / 2 - 2.0)
        shift = -8.0 + 8.0 * i / max(1, n_rep - 1)
        out.append(protein_system(seed=seed * 1000 + i, n_atoms=n, box=box, radius=radius, mcsteps=mcsteps,
                                  conf_bias=conf_bias, muex_shift=shift))
    return out


def slab_system(seed: int = 1, n_atoms: int = 200_000, box=(150.0, 150.0, 120.0), density: float = 0.09,
                pore: float = 12.0, n_frag: int = 8, n_types: int = 24, water: bool = True, mcsteps: int = 100_000,
                conf_bias: int = 1000, conc: float = 0.25, water_conc: float = 55.0, cutoff: float = 12.0,
                grid_dx: float = 1.0, excl: float = 1.6, water_fill: float = 1.0) -> System:
    """Large periodic system: a slab of random-walk chains with a cylindrical pore
    along z, generic rigid fragments and (optionally) TIP3P water.

    The slab holds ``n_atoms`` at ``density`` atoms/A^3, so its thickness is
    n_atoms / (density * (Lx Ly - pi pore^2)); chains restart at a random free
    point when a step cannot be placed.  LJ types, charges and fragment
    templates are drawn as in :func:`protein_system`; water is the TIP3P model
    (O -0.834, eps 0.1521, rmin/2 1.7682; H +0.417, eps 0.046, rmin/2 0.2245)
    named ``SOL`` (equal move probabilities), with ``water_fill`` times its
    bulk count (``water_conc`` mol/L over the volume outside the slab) placed
    initially, >= 2.2 A from everything.
    """
    g = np.random.default_rng(seed)
    L = np.asarray(box, dtype=np.float64)
    area = L[0] * L[1] - math.pi * pore * pore
    thick = n_atoms / (density * area)
    if thick >= L[2]:
        raise ValueError("slab thicker than the box")
    xyz = np.empty((n_atoms, 3), dtype=np.float32)
    nbreak = ctypes.c_int(0)
    rc = lib().gcmc_synth_chain_slab(n_atoms, 0.0, float(L[0]), 0.0, float(L[1]), float(L[2] / 2), float(thick / 2),
                                     float(L[0] / 2), float(L[1] / 2), float(pore), 1.5, excl, int(seed) * 7919 + 29,
                                     ptr(xyz), ctypes.byref(nbreak))
    if rc != 0:
        raise RuntimeError("slab generation failed")
    tnames = [f"T{i:02d}" for i in range(n_types)]
    eps = g.uniform(0.02, 0.20, n_types)
    rmin2 = g.uniform(1.0, 2.2, n_types)
    nb = {tnames[i]: charmm_to_nb(eps[i], rmin2[i]) for i in range(n_types)}
    nb["OT"] = charmm_to_nb(0.1521, 1.7682)
    nb["HT"] = charmm_to_nb(0.046, 0.2245)
    q = g.normal(0.0, 0.35, n_atoms)
    q -= q.mean()
    ptype = g.integers(n_types, size=n_atoms)
    names, raw = [], []
    for f in range(n_frag):
        ns = int(g.integers(4, 13))
        kind = "planar" if g.random() < 0.5 else "tetrahedral"
        txyz = lattice_template(g, ns, kind)
        tq = g.normal(0.0, 0.3, ns)
        tq += (int(g.integers(-1, 2)) - tq.sum()) / ns
        raw.append((txyz, tq, [tnames[t] for t in g.integers(n_types, size=ns)]))
        names.append(f"FR{f:02d}")
    if water:
        raw.append((tip3p_template(), np.array([-0.834, 0.417, 0.417]), ["OT", "HT", "HT"]))
        names.append("SOL")
    t1, t2, ff = lj_pair_table([t for (_, _, tt) in raw for t in tt], [tnames[t] for t in ptype], nb)
    col = {t: i for i, t in enumerate(t2)}
    templates = [{"xyz": txyz, "q": tq, "type": np.array([col[t] for t in tt])} for (txyz, tq, tt) in raw]
    fixed_type = np.array([col[tnames[t]] for t in ptype])
    nt = len(names)
    muex = g.uniform(-5.0, -1.0, n_frag).tolist() + ([-5.8] if water else [])
    concs = [conc] * n_frag + ([water_conc] if water else [])
    free = float(np.prod(L)) - thick * area
    existing = np.ascontiguousarray(xyz, dtype=np.float32)
    lo = np.zeros(3, np.float32)
    Lf = L.astype(np.float32)
    initial = []
    for f in range(nt):
        n0 = int(round(concs[f] * free * V.MOLES_TO_MOLECULES * (water_fill if names[f] == "SOL" else 1.0)))
        tx = np.ascontiguousarray(templates[f]["xyz"] - templates[f]["xyz"].mean(axis=0), dtype=np.float32)
        out = np.zeros((n0, len(tx), 3), np.float32)
        if n0:
            rc = lib().gcmc_synth_place(len(existing), ptr(existing), ptr(lo), ptr(Lf), ptr(tx), len(tx), n0,
                                        2.2 if names[f] == "SOL" else 2.0, int(seed) * 104729 + 31 * f + 11, ptr(out))
            if rc != 0:
                raise RuntimeError("could not place the initial copies")
            existing = np.ascontiguousarray(np.concatenate([existing, out.reshape(-1, 3)]))
        initial.append([out[c].astype(np.float64) for c in range(n0)])
    start, grid, cav, dx = cavity_grid(existing.astype(np.float64), L, grid_dx)
    groups = fix_groups(xyz, 6.0)
    moves = move_array_np(mcsteps, names, [1.0] * nt, seed=seed + 1)
    s = assemble(names=names, templates=templates, initial=initial, fixed_xyz=xyz, fixed_q=q, fixed_type=fixed_type,
                 fixed_group=groups, muex=muex, conc=concs, conf_bias=[conf_bias] * nt, mctime=[1.0] * nt, cryst=L,
                 cutoff=cutoff, grid_dx=dx, start=start, grid=grid, cavity_factor=cav, ff=ff,
                 n_frag_types_ff=len(t1), n_types_ff=len(t2), moves=moves, seed=seed)
    s.grid_bits = cavity_bits(existing.astype(np.float64), L, grid_dx)
    s.meta.update({"chain_breaks": int(nbreak.value), "n_fixed": n_atoms, "box": tuple(L), "slab_thickness": thick,
                   "lj_types": {"names": list(t2),
                                "eps_kcal": np.array([(eps[tnames.index(n)] if n in tnames else
                                                       {"OT": 0.1521, "HT": 0.046}[n]) for n in t2]),
                                "rmin_half": np.array([(rmin2[tnames.index(n)] if n in tnames else
                                                        {"OT": 1.7682, "HT": 0.2245}[n]) for n in t2])}})
    return s
