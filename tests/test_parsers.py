"""Input readers against pyGCMC's own parsers on the synthetic files in
tests/golden/inputs/ (golden outputs made by tests/golden/make_parser_golden.py)."""
import json
import os

from conftest import ROOT

DIR = os.path.join(ROOT, "tests", "golden", "inputs")
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "parsers.json")))


def test_pdb():
    from pygcmc_b200.inputs import read_pdb
    for name in ("small.pdb", "nocryst.pdb"):
        cryst, at, _ = read_pdb(os.path.join(DIR, name))
        g = GOLD[name]
        assert cryst == g["cryst"]
        assert len(at) == len(g["atoms"])
        for k, a in enumerate(g["atoms"]):
            assert [at.serial[k], at.name[k], at.residue[k], at.sequence[k]] == a[:4]
            assert list(at.xyz[k]) == a[4:7]
            assert at.lines[k] == a[7]


def test_itp_top_psf_ff():
    from pygcmc_b200.inputs import read_ff, read_itp, read_psf, read_top
    assert read_itp(os.path.join(DIR, "frag.itp")) == GOLD["frag.itp"]
    atoms, _ = read_top(os.path.join(DIR, "system.top"))
    assert atoms == GOLD["system.top"]
    assert read_psf(os.path.join(DIR, "small.psf")) == GOLD["small.psf"]
    nb, nbfix = read_ff(os.path.join(DIR, "params.ff"))
    assert nb == GOLD["params.ff"]["nb"]
    assert [[a, b, v] for (a, b), v in nbfix.items()] == GOLD["params.ff"]["nbfix"]
