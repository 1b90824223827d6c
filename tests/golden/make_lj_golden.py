"""Golden output of pyGCMC's own type tables and LJ pair table
(GCMCSimulation.get_simulation, gcmc/python/simulation.py:37-86), run on a
synthetic set of fragment and environment atoms.

    python tests/golden/make_lj_golden.py /path/to/pyGCMC     (or PYGCMC_REFERENCE=...)

The reference module is loaded straight from the source tree (nothing is
copied).  get_simulation runs unmodified on an object whose file-reading,
move, grid, grouping and packing steps (the calls before and after the table
loop) are no-ops, so what it computes here is exactly the table loop's output:
atomtypes1, atomtypes2, ff_pairs and every atom's typeNum.  Writes
tests/golden/lj_table.json; tests/test_builders.py checks
pygcmc_b200.system.lj_pair_table against it.
"""
import importlib.util
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    spec = importlib.util.spec_from_file_location("gcmc_reference_simulation",
                                                  os.path.join(ref, "gcmc", "python", "simulation.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)

    class Run(mod.GCMCSimulation):
        def _skip(self):
            pass
        get_fragment = get_forcefield = get_move = get_grid = show_parameters = set_fixCut = update_data = _skip

    g = np.random.default_rng(11)
    names = [f"T{i:02d}" for i in range(9)] + ["OT", "HT"]
    nb = {n: [float(g.uniform(0.1, 0.4)), float(g.uniform(0.05, 1.0))] for n in names}
    # NBFIX pairs, stored in either order (the loop looks both up)
    nbfix = {("T01", "T05"): [0.21, 0.33], ("T07", "T02"): [0.27, 0.44], ("OT", "T03"): [0.31, 0.52]}
    frag_types = [["OT", "HT", "HT"], ["T01", "T02", "T01", "T07"], ["T05", "T03", "HT"]]
    env_types = ["T04", "T03", "T00", "T06", "T04", "T08", "T05", "T00", "OT"]
    o = Run()
    o.pdb_file, o.top_file, o.psf_file = "x.pdb", "x.top", None
    o.fragments = [[types.SimpleNamespace(type=t) for t in ft] for ft in frag_types]
    o.fragmentName = ["SOL", "FRA", "FRB"]
    o.atoms = [types.SimpleNamespace(type=t, residue="PRO") for t in env_types]
    o.nb_dict = {k: tuple(v) for k, v in nb.items()}
    o.nbfix_dict = {k: tuple(v) for k, v in nbfix.items()}
    o.get_simulation()
    out = {
        "nb": nb, "nbfix": [[a, b, v[0], v[1]] for (a, b), v in nbfix.items()],
        "frag_types": frag_types, "env_types": env_types,
        "ref_atomtypes1": o.atomtypes1, "ref_atomtypes2": o.atomtypes2,
        "ref_ff_pairs": [[float(x) for x in p] for p in o.ff_pairs],
        "ref_env_typenum": [a.typeNum for a in o.atoms],
        "ref_frag_typenum": [[a.typeNum for a in f] for f in o.fragments],
    }
    with open(os.path.join(HERE, "lj_table.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote lj_table.json")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYGCMC_REFERENCE")
    if not ref:
        sys.exit("usage: make_lj_golden.py /path/to/pyGCMC (or set PYGCMC_REFERENCE)")
    main(ref)
