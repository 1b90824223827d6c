"""Wall time of pyGCMC's own Python input builders (get_grid, set_fixCut,
update_data -- gcmc/python/dataset.py:21-373) against the C++ builders of
pygcmc_b200 on the same large synthetic system (the slab system: 200 000
fixed atoms, 8 fragment types and TIP3P water in a 150 x 150 x 120 A box).

    python tests/golden/time_ref_builders.py [/path/to/pyGCMC] [n_fixed]

Runs on the CPU only; prints one JSON line.  The reference modules are loaded
from its source tree as in make_builder_golden.py; the Python objects they read
are built before the clock starts.
"""
import json
import os
import random
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from make_builder_golden import A, load_reference  # noqa: E402


def main(ref, n_fixed):
    from pygcmc_b200 import system as S
    s = S.slab_system(n_atoms=n_fixed, mcsteps=1000, water_fill=1.0 if n_fixed >= 200_000 else 0.2)
    nfix = int(s.meta["n_fixed"])
    fix = s.atomInfo[:nfix]
    fr = s.fragmentInfo
    names = [n.decode().strip() for n in fr["name"]]
    tpl = [fr[i]["atoms"][: int(fr[i]["num_atoms"])] for i in range(len(fr))]
    copies = []
    for i in range(len(fr)):
        cs = []
        for j in range(int(fr[i]["totalNum"])):
            r = s.residueInfo[int(fr[i]["startRes"]) + j]
            cs.append(s.atomInfo[int(r["atomStart"]): int(r["atomStart"]) + int(r["atomNum"])])
        copies.append(cs)
    occupied = np.concatenate([fix["position"]] + [c["position"] for cs in copies for c in cs]).astype(np.float64)
    cryst = [float(c) for c in s.SimInfo[0]["cryst"]]
    fix_xyz = fix["position"].astype(np.float64)
    out = {"n_fixed": nfix, "n_atoms_total": int(s.SimInfo[0]["totalAtomNum"]),
           "n_residues": int(s.SimInfo[0]["totalResNum"])}

    # ours (C++ through the Python API)
    t0 = time.perf_counter()
    start, grid, cav, dx = S.cavity_grid(occupied, cryst, 1.0)
    t1 = time.perf_counter()
    groups = S.fix_groups(fix_xyz, 6.0)
    t2 = time.perf_counter()
    templates = [{"xyz": t["position"].astype(np.float64), "q": t["charge"], "type": t["type"]} for t in tpl]
    initial = [[c["position"].astype(np.float64) for c in cs] for cs in copies]
    S.assemble(names=names, templates=templates, initial=initial, fixed_xyz=fix_xyz, fixed_q=fix["charge"],
               fixed_type=fix["type"], fixed_group=groups, muex=list(fr["muex"]), conc=list(fr["conc"]),
               conf_bias=list(fr["confBias"]), mctime=list(fr["mcTime"]), cryst=cryst, cutoff=12.0, grid_dx=dx,
               start=start, grid=grid, cavity_factor=cav, ff=s.ff, n_frag_types_ff=int(s.SimInfo[0]["ffXNum"]),
               n_types_ff=int(s.SimInfo[0]["ffYNum"]), moves=s.moveArray, seed=1)
    t3 = time.perf_counter()
    out["ours_s"] = {"get_grid": t1 - t0, "set_fixCut": t2 - t1, "update_data": t3 - t2}

    # the reference's Python
    mods = load_reference(ref)
    D = mods["dataset"].GCMCDataset
    o = types.SimpleNamespace()
    o.atoms = [A(*p) for p in occupied]
    o.cryst = cryst
    o.cavity_bias = True
    o.grid_dx = 1.0
    t0 = time.perf_counter()
    D.get_grid(o)
    t1 = time.perf_counter()
    o.fix_atoms = [A(*p, charge=float(a["charge"]), typeNum=int(a["type"])) for p, a in zip(fix_xyz, fix)]
    o.fixCutoff = 6.0
    t1b = time.perf_counter()
    D.set_fixCut(o)
    t2 = time.perf_counter()
    o.fragmentName = names
    o.moveArray = s.moveArray
    o.fragments = [[A(*a["position"], charge=float(a["charge"]), typeNum=int(a["type"])) for a in t] for t in tpl]
    o.fraglist = [[[A(*a["position"], charge=float(a["charge"]), typeNum=int(a["type"])) for a in c] for c in cs]
                  for cs in copies]
    o.fragmuex = list(fr["muex"])
    o.fragconc = list(fr["conc"])
    o.fragconf = list(fr["confBias"])
    o.mctime = list(fr["mcTime"])
    o.volume = cryst[0] * cryst[1] * cryst[2]
    ffp = s.ff.reshape(-1, 2)
    o.ff_pairs = [[float(a), float(b)] for a, b in ffp]
    o.atomtypes1 = [str(i) for i in range(int(s.SimInfo[0]["ffXNum"]))]
    o.atomtypes2 = [str(i) for i in range(int(s.SimInfo[0]["ffYNum"]))]
    o.cutoff = 12.0
    o.showInfo = 0
    o.PME = 0
    o.mcsteps = len(s.moveArray)
    o.moveArray_n = np.bincount(s.moveArray, minlength=4 * len(names)).tolist()  # as get_move leaves it
    random.seed(1)
    t2b = time.perf_counter()
    D.update_data(o)
    t3 = time.perf_counter()
    out["reference_python_s"] = {"get_grid": t1 - t0, "set_fixCut": t2 - t1b, "update_data": t3 - t2b}
    print(json.dumps(out))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference", int(sys.argv[2]) if len(sys.argv) > 2 else 200_000)
