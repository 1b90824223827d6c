"""Output writers: the PDB snapshot and topology counts of pyGCMC's get_data
(gcmc/python/dataset.py:375-440).

:func:`pdb_string` returns the reference's PDB text for a state: the CRYST1
record, the fixed atoms' own input lines, one ATOM record per atom of every
occupied fragment slot (formatted in C++, ``gcmc_pdb_fragment_lines``), and
END.  :func:`topology_counts` rewrites the ``[ molecules ]`` section of a
GROMACS topology with the current fragment counts.
"""
import ctypes
import re

import numpy as np

from ._native import lib, ptr


def pdb_string(system, fixed_lines, atom_names, last_serial=None, last_residue=None) -> str:
    """PDB text of ``system``'s current state.

    ``fixed_lines``: the fixed atoms' PDB lines (without newlines), written as
    given; ``atom_names[t][k]``: atom names of fragment type t's sites;
    ``last_serial`` / ``last_residue``: the last fixed atom's serial and residue
    number (the fragment records continue from them + 1; 1 when absent).
    """
    cr = system.SimInfo[0]["cryst"]
    head = "CRYST1  %.3f  %.3f  %.3f  90.00  90.00  90.00 P 1           1\n" % (cr[0], cr[1], cr[2])
    body = "".join(line + "\n" for line in fixed_lines)
    nt = len(system.fragmentInfo)
    names = np.zeros((nt, 20, 4), dtype="S1")
    for t in range(nt):
        for k, nm in enumerate(atom_names[t]):
            b = nm.encode()[:4].ljust(4, b"\0")
            for c in range(4):
                names[t, k, c] = b[c:c + 1]
    names = np.ascontiguousarray(names)
    s0 = int(last_serial) + 1 if last_serial is not None else 1
    r0 = int(last_residue) + 1 if last_residue is not None else 1
    L = lib()
    args = (nt, ptr(system.fragmentInfo), ptr(system.residueInfo), ptr(system.atomInfo), ptr(names), s0, r0)
    need = L.gcmc_pdb_fragment_lines(*args, None, 0)
    if need < 0:
        raise ValueError("gcmc_pdb_fragment_lines")
    buf = ctypes.create_string_buffer(int(need) + 1)
    n = L.gcmc_pdb_fragment_lines(*args, buf, int(need))
    if n < 0:
        raise ValueError("gcmc_pdb_fragment_lines")
    frag = buf.raw[:n].decode().replace("\0", " ")
    return head + body + frag + "END\n"


def topology_counts(top: str, names, counts) -> str:
    """The topology text with its ``[ molecules ]`` entries for ``names`` set to
    ``counts`` (entries missing there are appended), laid out as get_data
    writes them (dataset.py:411-436)."""
    pieces = re.split(r"\[\s*molecules\s*\]", top)
    if len(pieces) < 2:
        raise ValueError("topology has no [ molecules ] section")
    section = pieces[1].strip() + "\n"
    current = {}
    for name, cnt in re.findall(r"(\S+?)\s+(\d+)", section):
        current[name] = cnt
    for name, n in zip(names, counts):
        if name in current:
            section = re.sub(r"%s\s+%s" % (re.escape(name), current[name]), "%s\t%d" % (name, int(n)), section)
        else:
            section += "%s\t%d\n" % (name, int(n))
    return pieces[0] + "\n[ molecules ]\n" + section
