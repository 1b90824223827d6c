"""Golden outputs of pyGCMC's own input builders (get_grid, get_move, set_fixCut,
update_data -- gcmc/python/dataset.py:21-373), run on a small seeded system.

    python tests/golden/make_builder_golden.py [/path/to/pyGCMC]

The reference modules are loaded straight from the source tree into a synthetic
package (nothing is copied); their methods run on a plain object carrying the
attributes they read.  Writes tests/golden/builders.npz (inputs and outputs);
tests/test_builders.py checks pygcmc_b200.system against it.
"""
import importlib.util
import os
import random
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(ref):
    pkg = types.ModuleType("gcmc_reference")
    pkg.__path__ = []
    sys.modules["gcmc_reference"] = pkg
    mods = {}
    for name in ("values", "dataset"):
        spec = importlib.util.spec_from_file_location(f"gcmc_reference.{name}",
                                                      os.path.join(ref, "gcmc", "python", f"{name}.py"))
        m = importlib.util.module_from_spec(spec)
        sys.modules[spec.name] = m
        spec.loader.exec_module(m)
        mods[name] = m
    return mods


class A:  # the atom objects of gcmc/python/protein_data.py carry these fields
    def __init__(self, x, y, z, charge=0.0, typeNum=0):
        self.x, self.y, self.z, self.charge, self.typeNum = x, y, z, charge, typeNum


def main(ref):
    mods = load_reference(ref)
    g = np.random.default_rng(5)
    # fixed atoms: a short random walk; fragments: two templates, a few copies of one
    n_fix = 400
    steps = g.normal(size=(n_fix, 3))
    steps *= 1.5 / np.linalg.norm(steps, axis=1)[:, None]
    fix = np.cumsum(steps, axis=0) + 20.0
    fix_q = g.normal(0, 0.3, n_fix)
    fix_t = g.integers(2, 6, n_fix)
    tpl = [np.array([[0.0, 0, 0], [1.4, 0, 0], [0.7, 1.2, 0]]), np.array([[0.0, 0, 0], [1.4, 0, 0], [2.1, 1.2, 0], [3.5, 1.2, 0]])]
    tpl_q = [np.array([-0.6, 0.3, 0.3]), np.array([0.1, -0.2, 0.2, -0.1])]
    tpl_t = [np.array([0, 1, 1]), np.array([0, 1, 0, 1])]
    copies = [[tpl[0] + c for c in (np.array([5.0, 6.0, 7.0]), np.array([30.0, 31.0, 8.0]))], []]
    cryst = [40.0, 40.0, 40.0]
    names = ["WAT3", "LIN4"]

    o = types.SimpleNamespace()
    o.atoms = [A(*p) for p in fix] + [A(*p) for c in copies[0] for p in c]
    o.cryst = cryst
    o.cavity_bias = True
    o.grid_dx = 1.0
    mods["dataset"].GCMCDataset.get_grid(o)
    random.seed(1234)
    o.fragmentName = names
    o.mctime = [1.0, 2.0]
    o.mcsteps = 500
    o.attempt_prob_frag = [0.3, 0.3, 0.2, 0.2]
    o.attempt_prob_water = [0.25, 0.25, 0.25, 0.25]
    mods["dataset"].GCMCDataset.get_move(o)
    o.fix_atoms = [A(*p, charge=q, typeNum=int(t)) for p, q, t in zip(fix, fix_q, fix_t)]
    o.fixCutoff = 6.0
    mods["dataset"].GCMCDataset.set_fixCut(o)
    groups = np.array([a.sequence2 for a in o.fix_atoms])
    o.fragments = [[A(*p, charge=q, typeNum=int(t)) for p, q, t in zip(tpl[i], tpl_q[i], tpl_t[i])] for i in range(2)]
    o.fraglist = [[[A(*p, charge=q, typeNum=int(t)) for p, q, t in zip(c, tpl_q[0], tpl_t[0])] for c in copies[0]], []]
    o.fragmuex = [-5.0, -2.0]
    o.fragconc = [55.0, 0.25]
    o.fragconf = [16, 8]
    o.volume = cryst[0] * cryst[1] * cryst[2]
    o.ff_pairs = [[0.3 + 0.01 * i, 0.5 + 0.02 * i] for i in range(2 * 6)]
    o.atomtypes1 = ["A", "B"]
    o.atomtypes2 = ["A", "B", "C", "D", "E", "F"]
    o.cutoff = 12.0
    o.showInfo = 0
    o.PME = 0
    mods["dataset"].GCMCDataset.update_data(o)
    # get_data (dataset.py:375-440): PDB of the fixed atoms' own lines plus the
    # fragments, and the [ molecules ] counts of the topology
    for k, a in enumerate(o.fix_atoms):
        a.serial = k + 1
        a.sequence = int(groups[k]) + 1
        a.s = "ATOM  %5d  CA  GLY A%4d    %8.3f%8.3f%8.3f  1.00  0.00" % (k + 1, int(groups[k]) + 1, a.x, a.y, a.z)
    frag_names = [["OW", "HW1", "HW2"], ["C1", "C2", "C3", "C4"]]
    for i in range(2):
        for k, a in enumerate(o.fragments[i]):
            a.name = frag_names[i][k]
    o.fragmentInfo[0]["totalNum"] = 2
    o.topologyType = "top"
    o.TOPString = "[ system ]\ntest\n\n[ molecules ]\nProtein 1\nWAT3 7\n"
    mods["dataset"].GCMCDataset.get_data(o)
    pdb, top = o.PDBString, o.TOPString
    np.savez_compressed(
        os.path.join(HERE, "builders.npz"),
        fix=fix, fix_q=fix_q, fix_t=fix_t, cryst=np.array(cryst),
        tpl0=tpl[0], tpl1=tpl[1], tpl_q0=tpl_q[0], tpl_q1=tpl_q[1], tpl_t0=tpl_t[0], tpl_t1=tpl_t[1],
        copies0=np.array(copies[0]), ff=np.array(o.ff, np.float32),
        ref_startxyz=np.array(o.startxyz), ref_grid=o.grid, ref_cavity=np.array(o.cavity_bias_factor),
        ref_moves=o.moveArray, ref_groups=groups, ref_frag=o.fragmentInfo, ref_res=o.residueInfo,
        ref_atoms=o.atomInfo, ref_info=o.SimInfo, ref_pdb=np.array(pdb), ref_top=np.array(top),
        frag_atom_names0=np.array(frag_names[0]), frag_atom_names1=np.array(frag_names[1]))
    print("wrote builders.npz")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYGCMC_REFERENCE")
    if not ref:
        sys.exit(f"usage: {os.path.basename(__file__)} /path/to/pyGCMC (or set PYGCMC_REFERENCE)")
    main(ref)
