"""The CPU oracle against the reference's known answers (no GPU).

Known answers come from the pyGCMC tree (fixture made by tests/golden/make_golden.py):
three-water insertion energies computed with OpenMM in test/jupyter/test2.ipynb
and the notebook's Rodrigues rotation example.
"""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "notebook_known_answers.json")))


def three_water_system(charges=True):
    from pygcmc_b200 import system as S
    p = GOLD["tip3p_nm_kJ"]
    nb = {"OT": (p["sigmaO"], p["epsilonO"]), "HT": (p["sigmaH"], p["epsilonH"])}
    t1, t2, ff = S.lj_pair_table(["OT", "HT", "HT"], [], nb)
    qO, qH = GOLD["tip3p_charges"]["O"], GOLD["tip3p_charges"]["H"]
    q = np.array([qO, qH, qH]) if charges else np.zeros(3)
    ws = [np.array(w) for w in GOLD["waters"]]
    cryst = np.array(GOLD["cryst"])
    start, grid, cav, dx = S.cavity_grid(np.concatenate(ws[:2]), cryst, 1.0)
    s = S.assemble(names=["SOL"], templates=[{"xyz": ws[0], "q": q, "type": np.array([0, 1, 1])}],
                   initial=[ws[:2]], fixed_xyz=np.zeros((0, 3)), fixed_q=np.zeros(0), fixed_type=np.zeros(0, int),
                   fixed_group=np.zeros(0, int), muex=[-5.6], conc=[55.0], conf_bias=[1], mctime=[1.0], cryst=cryst,
                   cutoff=GOLD["openmm_cutoff_A"], grid_dx=dx, start=start, grid=grid, cavity_factor=cav, ff=ff,
                   n_frag_types_ff=2, n_types_ff=2, moves=np.zeros(0, np.int32), seed=1)
    return s, ws


def insertion_energy(oracle, charges, mode=0):
    s, ws = three_water_system(charges)
    f = s.fragmentInfo[0]
    pose = ws[2].astype(np.float32)[None]
    c = pose[0].mean(axis=0)[None]
    e, ng, pairs = oracle.energy_batch(s, pose, f["atoms"]["charge"][:3], f["atoms"]["type"][:3], c, mode=mode)
    return e[0], ng[0], pairs


def test_three_water_lj_matches_openmm(oracle_lib):
    e, ng, pairs = insertion_energy(oracle_lib, charges=False)
    assert ng == 2 and pairs == 18
    # plain truncated LJ: same functional form as OpenMM's CutoffPeriodic LJ
    assert abs(e - GOLD["openmm_insert_dE_lj_only_kJ"]) < 5e-3


def test_three_water_coulomb_geometry(oracle_lib):
    """Coulomb part: the oracle's plain-cutoff term, and OpenMM's reaction-field
    term recomputed from the same pair geometry, match their references."""
    e_all, _, _ = insertion_energy(oracle_lib, charges=True)
    e_lj, _, _ = insertion_energy(oracle_lib, charges=False)
    ws = [np.array(w) for w in GOLD["waters"]]
    qO, qH = GOLD["tip3p_charges"]["O"], GOLD["tip3p_charges"]["H"]
    q = np.array([qO, qH, qH], dtype=np.float32).astype(np.float64)
    plain, rf = 0.0, 0.0
    rc, eps_rf = GOLD["openmm_cutoff_A"], 78.3
    k_rf = (eps_rf - 1) / (2 * eps_rf + 1) / rc ** 3
    c_rf = 1 / rc + k_rf * rc ** 2
    for other in ws[:2]:
        for i in range(3):
            for j in range(3):
                r = np.linalg.norm(ws[2][i].astype(np.float32).astype(np.float64) - other[j].astype(np.float32))
                plain += 1388.431112 * q[i] * q[j] / r
                rf += 1389.35456 * q[i] * q[j] * (1 / r + k_rf * r * r - c_rf)
    assert abs((e_all - e_lj) - plain) < 1e-9 * max(1.0, abs(plain))
    openmm_coul = GOLD["openmm_insert_dE_kJ"] - GOLD["openmm_insert_dE_lj_only_kJ"]
    assert abs(rf - openmm_coul) < 2e-3


def test_fp32_mirror_close(oracle_lib):
    e64, _, _ = insertion_energy(oracle_lib, charges=True, mode=0)
    e32, _, _ = insertion_energy(oracle_lib, charges=True, mode=1)
    assert abs(e32 - e64) < 1e-5 * abs(e64) + 1e-4


def test_rodrigues_known_answer(oracle_lib):
    r = GOLD["rodrigues"]
    v, R = oracle_lib.rotate_point(r["axis"], r["theta"], r["v"])
    np.testing.assert_allclose(v, r["v_rot"], atol=2e-7)
    np.testing.assert_allclose(R, np.array(r["R"]), atol=2e-7)


def test_det_sincos_accuracy(oracle_lib):
    xs = np.linspace(-2 * np.pi, 2 * np.pi, 4001).astype(np.float32)
    err = max(max(abs(oracle_lib.det_sincos(float(x))[0] - np.sin(np.float64(x))),
                  abs(oracle_lib.det_sincos(float(x))[1] - np.cos(np.float64(x)))) for x in xs)
    assert err < 4e-7


def test_philox_uniformity(oracle_lib):
    u = np.array([oracle_lib.philox([i, 7, 3 << 16, 0], [1, 0]) for i in range(4000)], dtype=np.float64)
    u = u.reshape(-1) / 2.0 ** 32
    assert abs(u.mean() - 0.5) < 0.01
    assert abs(u.var() - 1 / 12) < 0.005
    # different keys give different streams
    assert (oracle_lib.philox([0, 0, 0, 0], [1, 0]) != oracle_lib.philox([0, 0, 0, 0], [2, 0])).any()


@pytest.mark.parametrize("n", [1, 2, 3, 5, 17, 64, 100, 1000, 4097])
def test_perm_slot_is_permutation(oracle_lib, n):
    import ctypes
    opts = oracle_lib.options()
    slots = [oracle_lib.lib().or_perm_slot(ctypes.byref(opts), 11, 5, i, n) for i in range(n)]
    assert sorted(slots) == list(range(n))


def test_oracle_run_invariants(oracle_lib, protein_small):
    s = protein_small.copy()
    logs, E = oracle_lib.run(s, 60, threads=4)
    assert (logs["n_after"] <= s.fragmentInfo["maxNum"][logs["ftype"]]).all()
    # counts evolve consistently step to step
    for t in range(len(s.fragmentInfo)):
        sel = logs[logs["ftype"] == t]
        if len(sel) > 1:
            assert (sel["n_before"][1:] == sel["n_after"][:-1]).all()
    # deletes accept at most one, translate/rotate never change counts
    assert (logs["n_accept"][logs["move"] == 1] <= 1).all()
    m = logs["move"] >= 2
    assert (logs["n_before"][m] == logs["n_after"][m]).all()
