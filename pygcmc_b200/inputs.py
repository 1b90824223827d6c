"""Readers of pyGCMC's input formats (gcmc/python/protein_data.py:27-341):
PDB coordinates, GROMACS .top/.itp topologies, CHARMM .psf, and the GROMACS
force-field parameter file (.ff / .itp with [ atomtypes ], [ nonbond_params ],
[ pairtypes ]).

The accepted syntax and the fields taken are the reference's, so that a
pyGCMC input set reads the same here:

* PDB: CRYST1 gives the box (else the atoms' extent); ATOM/HETATM records
  longer than 54 characters give serial, name, residue, sequence (strings)
  and x, y, z from the fixed columns 31-54; the line itself is kept (it is
  written back unchanged by :func:`pygcmc_b200.writers.pdb_string`).
* Topology blocks: ``[ name ]`` headers; text after ``;`` or ``#`` on a line
  is dropped (directive lines such as ``#ifdef`` vanish, their contents stay).
  A molecule type's name is the first ``name number`` line of its
  [ moleculetype ] block and its atoms the lines of the first [ atoms ] block
  after it: ``nr type resnr residue atom cgnr charge`` -> (type, resnr,
  residue, atom, charge) as strings.
* .top: molecule types from the file, then from each ``#include "x.itp"``
  (outside ``#ifdef ... #endif``), in order; [ molecules ] lists
  ``name count``; the atom list repeats each molecule's first matching type.
* .psf: after the title block (its count line), the atom lines of the
  !NATOM block -> (type, resid, residue, name, charge).
* force field: [ atomtypes ] ``name at.num mass charge ptype sigma epsilon``
  -> sigma [nm], epsilon [kJ/mol]; [ nonbond_params ] and [ pairtypes ]
  ``i j func sigma epsilon`` -> pair overrides (a later entry for the same
  ordered pair replaces an earlier one, so [ pairtypes ] listed after
  [ nonbond_params ] win, as in the reference).

Include paths are resolved against the topology's directory.
"""
import os
import re
from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np

_HEADER = re.compile(r"\[(.*)\]")
_NAMED_COUNT = re.compile(r"(\w+)\s+(\d+)")
_TOP_ATOM = re.compile(r"(\d+)\s+(\S+)\s+(\d+)\s+(\S+)\s+(\S+)\s+(\d+)\s+([0-9\.\-]+)")
_PSF_ATOM = re.compile(r"^(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)")
_FF_ATOMTYPE = re.compile(r"(\S+)\s+(\S+)\s+([0-9\.\-]+)\s+([0-9\.\-]+)\s+(\S+)\s+([0-9\.\-]+)+\s+([0-9\.\-]+)")
_FF_PAIR = re.compile(r"(\S+)\s+(\S+)\s+([0-9\.\-]+)\s+([0-9\.\-]+)\s+([0-9\.\-]+)")
_INCLUDE = re.compile(r'^\s*#include "(.*?)"\s*$', re.MULTILINE)


@dataclass
class PdbAtoms:
    serial: List[str] = field(default_factory=list)
    name: List[str] = field(default_factory=list)
    residue: List[str] = field(default_factory=list)
    sequence: List[str] = field(default_factory=list)
    xyz: np.ndarray = None
    lines: List[str] = field(default_factory=list)

    def __len__(self):
        return len(self.lines)


def read_pdb(path) -> Tuple[List[float], PdbAtoms, str]:
    """(box edges, atoms, file text)."""
    text = open(path).read()
    lines = text.strip().split("\n")
    cryst = None
    for ln in lines:
        if ln.lower().startswith("cryst1 "):
            cryst = [float(v) for v in ln.split()[1:4]]
            break
    at = PdbAtoms()
    coords = []
    for ln in lines:
        head = ln[:6].lower()
        if (head.startswith("atom ") or head == "hetatm") and len(ln) > 54:
            coords.append((float(ln[30:38]), float(ln[38:46]), float(ln[46:54])))
            at.serial.append(ln[6:11].strip())
            at.name.append(ln[12:16].strip())
            at.residue.append(ln[17:20].strip())
            at.sequence.append(ln[22:26].strip())
            at.lines.append(ln)
    at.xyz = np.array(coords, dtype=np.float64).reshape(-1, 3)
    if cryst is None and len(at):
        cryst = [float(v) for v in at.xyz.max(axis=0) - at.xyz.min(axis=0)]
    return cryst, at, text


def topology_blocks(text: str):
    """[(block name, [content lines])] in file order; the first block is 'title'."""
    blocks = [("title", [])]
    for raw in text.split("\n"):
        ln = raw.split(";", 1)[0].split("#", 1)[0]
        m = _HEADER.match(ln)
        if m:
            blocks.append((m.group(1).strip(), []))
        elif ln.strip():
            blocks[-1][1].append(ln.strip())
    return blocks


def _molecule_types(blocks):
    """[(name, [atom tuples])] of every [ moleculetype ] block, in order."""
    out = []
    for b, (name, body) in enumerate(blocks):
        if name != "moleculetype":
            continue
        mname = None
        for ln in body:
            m = _NAMED_COUNT.match(ln)
            if m:
                mname = m.group(1)
                break
        if mname is None:
            continue
        atoms = []
        for name2, body2 in blocks[b + 1:]:
            if name2 == "atoms":
                for ln in body2:
                    m = _TOP_ATOM.match(ln)
                    if m:
                        atoms.append([m.group(2), m.group(3), m.group(4), m.group(5), m.group(7)])
                break
        out.append((mname, atoms))
    return out


def read_itp(path):
    """Atoms (type, resnr, residue, atom, charge) of the last molecule type in an .itp."""
    types = _molecule_types(topology_blocks(open(path).read()))
    return types[-1][1] if types else []


def read_top(path):
    """(atom list of the whole system, topology text)."""
    text = open(path).read()
    blocks = topology_blocks(text)
    stripped = re.sub(r"#ifdef .*?#endif", "", re.sub(r";.*", "", text), flags=re.DOTALL)
    base = os.path.dirname(os.path.abspath(path))
    types = _molecule_types(blocks)
    for inc in (x.strip() for x in _INCLUDE.findall(stripped)):
        if inc.endswith(".itp"):
            p = inc if os.path.isabs(inc) else os.path.join(base, inc)
            types += _molecule_types(topology_blocks(open(p).read()))
    molecules = []
    for name, body in blocks:
        if name == "molecules":
            for ln in body:
                m = _NAMED_COUNT.match(ln)
                if m:
                    molecules.append((m.group(1), int(m.group(2))))
            break
    atoms = []
    for mname, count in molecules:
        for tname, tatoms in types:
            if tname == mname:
                atoms += tatoms * count
                break
    return atoms, text


def _int_line(ln):
    try:
        return int(ln)
    except ValueError:
        return None


def read_psf(path):
    """Atoms (type, resid, residue, name, charge) of a CHARMM .psf."""
    lines = open(path).read().strip().split("\n")[1:]
    lines = [re.split(r"[*!#]", ln, maxsplit=1)[0] for ln in lines]

    def skip_to_count(seq):
        for i, ln in enumerate(seq):
            n = _int_line(ln)
            if n is not None:
                return i, n
        raise ValueError("psf: no count line")

    i, ntitle = skip_to_count(lines)
    lines = lines[i + ntitle + 1:]
    i, natom = skip_to_count(lines)
    out = []
    for ln in lines[i + 1:]:
        m = _PSF_ATOM.match(ln.strip())
        if m:
            if len(out) == natom:
                break
            out.append([m.group(6), m.group(3), m.group(4), m.group(5), m.group(7)])
    return out


def read_ff(path) -> Tuple[Dict[str, List[float]], Dict[Tuple[str, str], List[float]]]:
    """(per-type [sigma nm, epsilon kJ/mol], pair overrides {(i, j): [sigma, epsilon]})."""
    nb, nbfix = {}, {}
    for name, body in topology_blocks(open(path).read()):
        if name == "atomtypes":
            for ln in body:
                m = _FF_ATOMTYPE.match(ln)
                if m:
                    nb[m.group(1)] = [float(m.group(6)), float(m.group(7))]
        if name in ("nonbond_params", "pairtypes"):
            for ln in body:
                m = _FF_PAIR.match(ln)
                if m:
                    nbfix[(m.group(1), m.group(2))] = [float(m.group(4)), float(m.group(5))]
    return nb, nbfix
