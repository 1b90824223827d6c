"""Input builders against pyGCMC's own get_grid / get_move / set_fixCut /
update_data outputs (fixture: tests/golden/make_builder_golden.py)."""
import os
import random

import numpy as np
import pytest

from conftest import ROOT

FIX = os.path.join(ROOT, "tests", "golden", "builders.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(FIX)


def all_atoms(d):
    return np.concatenate([d["fix"]] + list(d["copies0"]))


def test_cavity_grid_matches_reference(gold):
    from pygcmc_b200.system import cavity_grid
    start, grid, cav, dx = cavity_grid(all_atoms(gold), gold["cryst"], 1.0)
    np.testing.assert_array_equal(np.array(start), gold["ref_startxyz"])
    assert cav == float(gold["ref_cavity"])
    mine = {tuple(p) for p in grid.reshape(-1, 3).tolist()}
    ref = {tuple(p) for p in gold["ref_grid"].reshape(-1, 3).tolist()}
    assert mine == ref and len(grid) == len(gold["ref_grid"])


def expand_bits(rec):
    """CPU expansion of a gcmc_grid_bits record: the marked voxels in increasing
    voxel index, each corner an FP64 product and sum rounded once to float."""
    start = np.frombuffer(rec[0:24].tobytes(), np.float64)
    dx = float(np.frombuffer(rec[24:32].tobytes(), np.float64)[0])
    n = np.frombuffer(rec[32:44].tobytes(), np.int32).astype(np.int64)
    words = np.frombuffer(rec[48:].tobytes(), np.uint32)
    bits = np.unpackbits(words.view(np.uint8), bitorder="little")[: n.prod()]
    v = np.flatnonzero(bits).astype(np.int64)
    x, r = np.divmod(v, n[1] * n[2])
    y, z = np.divmod(r, n[2])
    return np.stack([x * dx + start[0], y * dx + start[1], z * dx + start[2]], axis=1).astype(np.float32)


@pytest.mark.parametrize("bias,dx", [(True, 1.0), (True, 0.7), (False, 1.0)])
def test_cavity_bits_expand_to_the_float_grid(gold, bias, dx):
    from pygcmc_b200.system import cavity_bits, cavity_grid
    start, grid, cav, gdx = cavity_grid(all_atoms(gold), gold["cryst"], dx, cavity_bias=bias)
    rec = cavity_bits(all_atoms(gold), gold["cryst"], dx, cavity_bias=bias)
    assert rec.dtype == np.uint8
    np.testing.assert_array_equal(np.frombuffer(rec[0:24].tobytes(), np.float64), start)
    assert float(np.frombuffer(rec[24:32].tobytes(), np.float64)[0]) == gdx
    pts = expand_bits(rec)
    np.testing.assert_array_equal(pts.view(np.uint32), grid.reshape(-1, 3).view(np.uint32))


def test_cavity_bits_of_the_reference_grid(gold):
    from pygcmc_b200.system import cavity_bits
    pts = expand_bits(cavity_bits(all_atoms(gold), gold["cryst"], 1.0))
    assert {tuple(p) for p in pts.tolist()} == {tuple(p) for p in gold["ref_grid"].reshape(-1, 3).tolist()}
    assert len(pts) * 3 == len(gold["ref_grid"])


def test_builders_attach_the_bit_set(protein_small, water_small):
    for s in (protein_small, water_small):
        pts = expand_bits(s.grid_bits)
        assert len(pts) == int(s.SimInfo[0]["totalGridNum"])
        np.testing.assert_array_equal(pts.reshape(-1).view(np.uint32), s.grid.view(np.uint32))
        c = s.copy()
        assert c.grid_bits is not s.grid_bits and np.array_equal(c.grid_bits, s.grid_bits)


def test_move_schedule_matches_reference(gold):
    from pygcmc_b200.system import move_array
    mv = move_array(500, ["WAT3", "LIN4"], [1.0, 2.0], rng=random.Random(1234))
    np.testing.assert_array_equal(mv, gold["ref_moves"])


def test_fixed_groups_match_reference(gold):
    from pygcmc_b200.system import fix_groups
    np.testing.assert_array_equal(fix_groups(gold["fix"], 6.0), gold["ref_groups"])


def test_update_data_matches_reference(gold):
    from pygcmc_b200.system import assemble, cavity_grid, fix_groups
    d = gold
    start, grid, cav, dx = cavity_grid(all_atoms(d), d["cryst"], 1.0)
    tpl = [{"xyz": d["tpl0"], "q": d["tpl_q0"], "type": d["tpl_t0"]},
           {"xyz": d["tpl1"], "q": d["tpl_q1"], "type": d["tpl_t1"]}]
    s = assemble(names=["WAT3", "LIN4"], templates=tpl, initial=[list(d["copies0"]), []], fixed_xyz=d["fix"],
                 fixed_q=d["fix_q"], fixed_type=d["fix_t"], fixed_group=fix_groups(d["fix"], 6.0),
                 muex=[-5.0, -2.0], conc=[55.0, 0.25], conf_bias=[16, 8], mctime=[1.0, 2.0], cryst=d["cryst"],
                 cutoff=12.0, grid_dx=dx, start=start, grid=grid, cavity_factor=cav, ff=d["ff"], n_frag_types_ff=2,
                 n_types_ff=6, moves=d["ref_moves"], seed=0)
    rf, rr, ra, ri = d["ref_frag"], d["ref_res"], d["ref_atoms"], d["ref_info"]
    for f in ("name", "startRes", "muex", "conc", "confBias", "mcTime", "totalNum", "maxNum", "num_atoms"):
        np.testing.assert_array_equal(s.fragmentInfo[f], rf[f], err_msg=f)
    for i in range(2):
        n = int(rf[i]["num_atoms"])
        np.testing.assert_array_equal(s.fragmentInfo[i]["atoms"][:n], rf[i]["atoms"][:n])
    np.testing.assert_array_equal(s.residueInfo["atomNum"], rr["atomNum"])
    np.testing.assert_array_equal(s.residueInfo["atomStart"], rr["atomStart"])
    defined = list(range(int(rf[0]["startRes"])))  # fixed groups
    for i in range(2):
        defined += list(range(int(rf[i]["startRes"]), int(rf[i]["startRes"]) + int(rf[i]["totalNum"])))
    np.testing.assert_array_equal(s.residueInfo["position"][defined], rr["position"][defined])
    atoms = list(range(len(d["fix"])))
    for r in defined[int(rf[0]["startRes"]):]:
        atoms += list(range(int(rr[r]["atomStart"]), int(rr[r]["atomStart"]) + int(rr[r]["atomNum"])))
    np.testing.assert_array_equal(s.atomInfo[atoms], ra[atoms])
    for f in ("mcsteps", "cutoff", "grid_dx", "startxyz", "cryst", "cavityFactor", "fragTypeNum", "totalGridNum",
              "totalResNum", "totalAtomNum", "ffXNum", "ffYNum", "PME"):
        np.testing.assert_array_equal(s.SimInfo[0][f], ri[0][f], err_msg=f)


def test_lj_pair_table_combining_rules():
    """Lorentz-Berthelot unless an NBFIX pair exists (simulation.py:56-75)."""
    from pygcmc_b200.system import lj_pair_table
    nb = {"A": (0.3, 0.5), "B": (0.2, 0.8), "C": (0.35, 0.2)}
    t1, t2, ff = lj_pair_table(["A", "B", "A"], ["C", "A"], nb, nbfix={("C", "B"): (0.11, 0.22)})
    assert t1 == ["A", "B"] and t2 == ["A", "B", "C"]
    tab = ff.reshape(2, 3, 2)
    np.testing.assert_allclose(tab[0, 1], [(0.3 + 0.2) / 2, np.sqrt(0.5 * 0.8)], rtol=1e-6)
    np.testing.assert_allclose(tab[1, 2], [0.11, 0.22], rtol=1e-6)
    np.testing.assert_allclose(tab[0, 0], [0.3, 0.5], rtol=1e-6)


def test_lj_pair_table_matches_reference_get_simulation():
    """Type tables and pair table equal the output of pyGCMC's own get_simulation
    loop (simulation.py:37-86) on the golden case (tests/golden/make_lj_golden.py):
    row and column type order, NBFIX looked up in both orders, Lorentz-Berthelot
    otherwise, each atom's column index, and the float32 table bit for bit."""
    import json
    from pygcmc_b200.system import lj_pair_table
    with open(os.path.join(ROOT, "tests", "golden", "lj_table.json")) as f:
        G = json.load(f)
    nb = {k: tuple(v) for k, v in G["nb"].items()}
    nbfix = {(a, b): (s, e) for a, b, s, e in G["nbfix"]}
    frag_flat = [t for ft in G["frag_types"] for t in ft]
    t1, t2, ff = lj_pair_table(frag_flat, G["env_types"], nb, nbfix)
    assert t1 == G["ref_atomtypes1"] and t2 == G["ref_atomtypes2"]
    ref_ff = np.array(G["ref_ff_pairs"], dtype=np.float32).ravel()
    assert np.array_equal(ff, ref_ff)
    col = {t: i for i, t in enumerate(t2)}
    assert [col[t] for t in G["env_types"]] == G["ref_env_typenum"]
    assert [[col[t] for t in ft] for ft in G["frag_types"]] == G["ref_frag_typenum"]
