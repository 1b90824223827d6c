"""Output writers against pyGCMC's own get_data output (tests/golden/builders.npz,
made by tests/golden/make_builder_golden.py from the reference's dataset.py)."""
import os

import numpy as np

from conftest import ROOT

FIX = os.path.join(ROOT, "tests", "golden", "builders.npz")


def _state(d):
    from pygcmc_b200.system import System
    frag = d["ref_frag"].copy()
    frag[0]["totalNum"] = 2
    return System(d["ref_info"].copy(), frag, d["ref_res"].copy(), d["ref_atoms"].copy(),
                  np.zeros(3, np.float32), d["ff"], np.zeros(0, np.int32))


def test_pdb_matches_reference_get_data(native_lib):
    from pygcmc_b200.writers import pdb_string
    d = np.load(FIX)
    s = _state(d)
    fix, groups = d["fix"], d["ref_groups"]
    lines = ["ATOM  %5d  CA  GLY A%4d    %8.3f%8.3f%8.3f  1.00  0.00" % (k + 1, int(groups[k]) + 1, *fix[k])
             for k in range(len(fix))]
    names = [list(d["frag_atom_names0"]), list(d["frag_atom_names1"])]
    got = pdb_string(s, lines, names, last_serial=len(fix), last_residue=int(groups[-1]) + 1)
    assert got == str(d["ref_pdb"])


def test_topology_counts_match_reference(native_lib):
    from pygcmc_b200.writers import topology_counts
    d = np.load(FIX)
    top = "[ system ]\ntest\n\n[ molecules ]\nProtein 1\nWAT3 7\n"
    assert topology_counts(top, ["WAT3", "LIN4"], [2, 0]) == str(d["ref_top"])
