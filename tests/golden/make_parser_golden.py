"""Golden outputs of pyGCMC's own input parsers (read_pdb, read_itp, read_top,
read_psf, read_ff -- gcmc/python/protein_data.py:27-341) on the synthetic files
in tests/golden/inputs/.

    python tests/golden/make_parser_golden.py [/path/to/pyGCMC]

The reference module is loaded straight from its source tree (nothing is
copied).  read_top opens its #include files relative to the working
directory, so this runs inside tests/golden/inputs/.  Writes
tests/golden/parsers.json; tests/test_parsers.py checks pygcmc_b200.inputs
against it.
"""
import importlib.util
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    spec = importlib.util.spec_from_file_location("gcmc_reference_protein_data",
                                                  os.path.join(ref, "gcmc", "python", "protein_data.py"))
    P = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(P)
    cwd = os.getcwd()
    os.chdir(os.path.join(HERE, "inputs"))
    try:
        out = {}
        for name in ("small.pdb", "nocryst.pdb"):
            cryst, atoms, s = P.read_pdb(name)
            out[name] = {"cryst": cryst, "atoms": [[a.serial, a.name, a.residue, a.sequence, a.x, a.y, a.z, a.s]
                                                   for a in atoms]}
        out["frag.itp"] = P.read_itp("frag.itp")
        atoms_top, s = P.read_top("system.top")
        out["system.top"] = atoms_top
        out["small.psf"] = P.read_psf("small.psf")
        nb, nbfix = P.read_ff("params.ff")
        out["params.ff"] = {"nb": nb, "nbfix": [[a, b, v] for (a, b), v in nbfix.items()]}
    finally:
        os.chdir(cwd)
    with open(os.path.join(HERE, "parsers.json"), "w") as f:
        json.dump(out, f, indent=0)
    print("wrote parsers.json")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYGCMC_REFERENCE")
    if not ref:
        sys.exit(f"usage: {os.path.basename(__file__)} /path/to/pyGCMC (or set PYGCMC_REFERENCE)")
    main(ref)
