"""Generates the committed golden fixtures from the pyGCMC source tree.

    python tests/golden/make_golden.py [/path/to/pyGCMC]

Writes tests/golden/notebook_known_answers.json: the three-water coordinates of
test/water/3water.pdb and the numbers printed by test/jupyter/test2.ipynb
(OpenMM insertion energies, TIP3P parameters, Rodrigues rotation example).
The values are read from those files, not typed in.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def cell_text(nb, i):
    c = nb["cells"][i]
    src = "".join(c["source"])
    outs = []
    for o in c.get("outputs", []):
        if "text" in o:
            outs.append("".join(o["text"]))
        elif "data" in o and "text/plain" in o["data"]:
            outs.append("".join(o["data"]["text/plain"]))
    return src, "\n".join(outs)


def floats(s):
    return [float(x) for x in re.findall(r"-?\d+\.\d+(?:e-?\d+)?", s)]


def main(ref):
    waters = {}
    for line in open(os.path.join(ref, "test", "water", "3water.pdb")):
        if line.startswith("ATOM"):
            waters.setdefault(line[22:26], []).append(
                [float(line[30:38]), float(line[38:46]), float(line[46:54])])
        if line.startswith("CRYST1"):
            cryst = [float(line[6:15]), float(line[15:24]), float(line[24:33])]
    nb = json.load(open(os.path.join(ref, "test", "jupyter", "test2.ipynb")))
    e_full = floats(cell_text(nb, 9)[1])[0]       # E(3 waters) - E(2 waters), OpenMM, kJ/mol
    e_lj = floats(cell_text(nb, 13)[1])[0]        # same with charges zeroed
    params = floats(cell_text(nb, 14)[0])         # sigmaO, epsilonO, sigmaH, epsilonH
    rot_src, rot_out = cell_text(nb, 22)
    v_rot = floats(rot_out)
    r_src, r_out = cell_text(nb, 23)
    R = floats(r_out)
    axis = floats(re.search(r"k = np.array\(\[(.*?)\]\)", rot_src).group(1))
    theta = floats(re.search(r"theta = (.*)", rot_src).group(1))[0]
    v = floats(re.search(r"v = np.array\(\[(.*?)\]\)", rot_src).group(1))
    out = {
        "source": "test/water/3water.pdb; test/jupyter/test2.ipynb cells 9, 13, 14, 22, 23",
        "cryst": cryst,
        "waters": [waters[k] for k in waters],
        "openmm_insert_dE_kJ": e_full,
        "openmm_insert_dE_lj_only_kJ": e_lj,
        "openmm_cutoff_A": 15.0,
        "tip3p_nm_kJ": {"sigmaO": params[0], "epsilonO": params[1], "sigmaH": params[2], "epsilonH": params[3]},
        "tip3p_charges": {"O": -0.834, "H": 0.417},
        "rodrigues": {"axis": axis, "theta": theta, "v": v, "v_rot": v_rot, "R": [R[0:3], R[3:6], R[6:9]]},
    }
    with open(os.path.join(HERE, "notebook_known_answers.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote notebook_known_answers.json")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYGCMC_REFERENCE")
    if not ref:
        sys.exit(f"usage: {os.path.basename(__file__)} /path/to/pyGCMC (or set PYGCMC_REFERENCE)")
    main(ref)
