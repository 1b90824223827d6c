"""Edge cases against the oracle (needs a B200): empty and full fragment
types, the smallest and largest fragments (1 and 20 sites), the largest
confBias (1024), zero-step calls."""
import numpy as np
import pytest

from test_gpu_parity import check_trajectory, occupied_atoms

pytestmark = pytest.mark.gpu


def edge_system(seed=4, mcsteps=160, conf_bias=64, initial=(0, 2)):
    """A small random-walk 'protein' with a 1-site ion (charge +1) and a
    20-site planar fragment; `initial` copies of each are placed at start."""
    from pygcmc_b200 import system as S
    g = np.random.default_rng(seed)
    L = np.array([32.0, 32.0, 32.0])
    steps = g.normal(size=(600, 3))
    steps *= 1.5 / np.linalg.norm(steps, axis=1)[:, None]
    fix = np.cumsum(steps, axis=0) % L
    nb = {f"T{i}": S.charmm_to_nb(g.uniform(0.02, 0.2), g.uniform(1.0, 2.2)) for i in range(6)}
    big = S.lattice_template(g, 20, "planar")
    tq = g.normal(0, 0.3, 20)
    tq -= tq.mean()
    t1, t2, ff = S.lj_pair_table(["T0"] + [f"T{1 + i % 5}" for i in range(20)], ["T1", "T2", "T3"], nb)
    col = {t: i for i, t in enumerate(t2)}
    templates = [{"xyz": np.zeros((1, 3)), "q": np.array([1.0]), "type": np.array([col["T0"]])},
                 {"xyz": big, "q": tq, "type": np.array([col[f"T{1 + i % 5}"] for i in range(20)])}]
    init = []
    for f, n0 in enumerate(initial):
        init.append([templates[f]["xyz"] - templates[f]["xyz"].mean(axis=0) + g.random(3) * L for _ in range(n0)])
    allxyz = np.concatenate([fix] + [p for c in init for p in c])
    start, grid, cav, dx = S.cavity_grid(allxyz, L, 1.0)
    q = g.normal(0, 0.3, len(fix))
    q -= q.mean()
    moves = S.move_array_np(mcsteps, ["ION", "BIG"], [1.0, 1.0], seed=seed)
    return S.assemble(names=["ION", "BIG"], templates=templates, initial=init, fixed_xyz=fix, fixed_q=q,
                      fixed_type=np.array([col["T" + str(1 + i % 3)] for i in range(len(fix))]),
                      fixed_group=S.fix_groups(fix, 6.0), muex=[-3.0, -8.0], conc=[0.5, 0.05],
                      conf_bias=[conf_bias, conf_bias], mctime=[1.0, 1.0], cryst=L, cutoff=12.0, grid_dx=dx,
                      start=start, grid=grid, cavity_factor=cav, ff=ff, n_frag_types_ff=len(t1),
                      n_types_ff=len(t2), moves=moves, seed=seed)


def test_one_and_twenty_site_fragments_start_empty(oracle_lib, native_lib):
    s = edge_system(initial=(0, 0))
    logs = check_trajectory(oracle_lib, s, 160)
    assert (logs["n_accept"][logs["move"] == 0] > 0).any()  # insertions happened
    assert ((logs["move"] == 1) & (logs["n_before"] == 0)).any()  # deletes on an empty type were skipped
    assert (logs["k"][(logs["move"] >= 2) & (logs["n_before"] == 0)] == 0).all()


def test_full_fragment_type_skips_insertions(oracle_lib, native_lib):
    s = edge_system(initial=(3, 2))
    s.fragmentInfo[1]["maxNum"] = s.fragmentInfo[1]["totalNum"]  # type 1 full: insertions have no poses
    cap = int(s.fragmentInfo[1]["maxNum"])
    logs = check_trajectory(oracle_lib, s, 120)
    full = (logs["move"] == 0) & (logs["ftype"] == 1) & (logs["n_before"] >= cap)
    assert full.any() and (logs["k"][full] == 0).all()
    assert (logs["n_after"][logs["ftype"] == 1] <= cap).all()


def test_largest_conf_bias(oracle_lib, native_lib):
    s = edge_system(conf_bias=1024, mcsteps=40, initial=(2, 1))
    logs = check_trajectory(oracle_lib, s, 40)
    assert (logs["k"][logs["move"] == 0] == 1024).any()


def test_zero_step_call_changes_nothing(native_lib, protein_small):
    from pygcmc_b200.gpu import runGCMC
    s = protein_small.copy()
    before = s.copy()
    s.SimInfo[0]["mcsteps"] = 0
    runGCMC(*s.arrays())
    assert np.array_equal(s.atomInfo, before.atomInfo)
    assert np.array_equal(s.residueInfo, before.residueInfo)
    assert (s.fragmentInfo["totalNum"] == before.fragmentInfo["totalNum"]).all()
