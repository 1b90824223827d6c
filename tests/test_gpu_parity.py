"""CUDA engine vs the CPU oracle on the same seeded inputs (needs a B200).

* pose energies: FP64 sums of FP32 pair terms on the GPU vs the oracle's FP64
  restatement of calcEnergy, per pose within 1e-5 relative or 1e-4 kcal/mol
  (relative to |E| for these poses), with bit-identical group-inclusion counts;
* trajectories: the oracle replays the engine's logged energies; every step's
  move, pose count, cluster count, accepts, first accepted pose and counts
  must be identical, the oracle's own FP64 energies must agree with the
  engine's within 1e-5 of the sum of |pair terms| (both energies' pairs for a
  translate/rotate dE) or 1e-4 kcal/mol, and the final coordinates of every
  occupied slot must be bit-identical.
"""
import numpy as np
import pytest

from conftest import energy_close

pytestmark = pytest.mark.gpu

LOG_KMAX = 1024
LOG_FIELDS = ("step", "move", "ftype", "k", "n_before", "n_after", "n_clusters", "n_accept", "first_accept", "slot")


def engine_trajectory(system, nsteps, **opt):
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    opts = default_options(log_steps=nsteps, log_kmax=LOG_KMAX, **opt)
    with Engine(system.copy(), opts) as eng:
        eng.run(nsteps)
        eng.sync()
        logs, E = eng.logs()
        final = eng.download()
        counters = eng.counters()
    return logs, E, final, counters


def occupied_atoms(s):
    idx = []
    for f in s.fragmentInfo:
        for j in range(int(f["totalNum"])):
            r = s.residueInfo[int(f["startRes"]) + j]
            idx.extend(range(int(r["atomStart"]), int(r["atomStart"]) + int(r["atomNum"])))
    return np.array(idx, dtype=np.int64)


def occupied_res(s):
    return np.concatenate([np.arange(int(f["startRes"]), int(f["startRes"]) + int(f["totalNum"]))
                           for f in s.fragmentInfo])


def check_trajectory(oracle, system, nsteps, proposal=0, muex_kcal=0, **engine_opts):
    logs_g, E_g, final_g, counters = engine_trajectory(system, nsteps, proposal=proposal, muex_kcal=muex_kcal,
                                                       **engine_opts)
    assert len(logs_g) == nsteps
    s_o = system.copy()
    opts = oracle.options(proposal=proposal, muex_kcal=muex_kcal)
    r = oracle.run_ext(s_o, nsteps, opts=opts, kmax=LOG_KMAX, replay=E_g)
    logs_o, E_o, SC = r["logs"], r["energies"], r["scale"]
    for f in LOG_FIELDS:
        bad = np.flatnonzero(logs_g[f] != logs_o[f])
        assert bad.size == 0, (f, bad[:5], logs_g[bad[:3]], logs_o[bad[:3]])
    # the running energy (FP64 sum of the accepted energy changes) is the same sum
    assert np.array_equal(logs_g["e_total"], logs_o["e_total"])
    mask = np.arange(LOG_KMAX)[None, :] < logs_g["k"][:, None]
    ok = energy_close(E_g[mask], E_o[mask], SC[mask])
    assert ok.all(), (np.flatnonzero(~ok)[:10], E_g[mask][~ok][:5], E_o[mask][~ok][:5])
    rel = np.abs(E_g[mask] - E_o[mask]) / np.maximum(SC[mask], 1e-30)
    print(f"max |dE err| / sum|pair terms| = {rel.max():.2e}")
    assert (final_g.fragmentInfo["totalNum"] == s_o.fragmentInfo["totalNum"]).all()
    a = occupied_atoms(s_o)
    assert np.array_equal(final_g.atomInfo["position"][a], s_o.atomInfo["position"][a])
    r = occupied_res(s_o)
    assert np.array_equal(final_g.residueInfo["position"][r], s_o.residueInfo["position"][r])
    assert counters["steps"] == nsteps
    return logs_g


def explicit_poses(oracle, system, per_type=64):
    """Insertion poses of every type plus the current pose of occupied slots."""
    out = []
    for t, f in enumerate(system.fragmentInfo):
        ns = int(f["num_atoms"])
        xyz, cen, self_res = [], [], []
        for i in range(per_type):
            p, c = oracle.insert_pose(system, t, 5, i)
            xyz.append(p)
            cen.append(c)
            self_res.append(-1)
        for j in range(min(int(f["totalNum"]), per_type)):
            r = system.residueInfo[int(f["startRes"]) + j]
            a0 = int(r["atomStart"])
            xyz.append(system.atomInfo["position"][a0:a0 + ns])
            cen.append(r["position"])
            self_res.append(int(f["startRes"]) + j)
        out.append((t, np.array(xyz, np.float32), np.array(cen, np.float32), np.array(self_res, np.int32),
                    f["atoms"]["charge"][:ns].copy(), f["atoms"]["type"][:ns].copy()))
    return out


@pytest.mark.parametrize("which", ["water_small", "protein_small"])
def test_pose_energies_match_oracle(request, oracle_lib, which):
    from pygcmc_b200.engine import Engine
    s = request.getfixturevalue(which)
    with Engine(s.copy()) as eng:
        for t, xyz, cen, self_res, q, ty in explicit_poses(oracle_lib, s):
            e_g, ng_g = eng.energy_poses(xyz, q, ty, cen, self_res)
            e_o, ng_o, _, l1 = oracle_lib.energy_batch(s, xyz, q, ty, cen, self_res, mode=0, want_l1=True)
            assert np.array_equal(ng_g, ng_o), (t, np.flatnonzero(ng_g != ng_o)[:5])
            ok = energy_close(e_g, e_o, l1) & energy_close(e_g, e_o)
            assert ok.all(), (t, e_g[~ok][:5], e_o[~ok][:5])


def test_trajectory_protein_reference_mode(oracle_lib, protein_small):
    logs = check_trajectory(oracle_lib, protein_small, 240)
    assert (logs["n_accept"] > 0).any()
    assert set(np.unique(logs["move"])) == {0, 1, 2, 3}


def test_trajectory_water_reference_mode(oracle_lib, water_small):
    check_trajectory(oracle_lib, water_small, 120)


def test_trajectory_protein_symmetric_mode(oracle_lib, protein_small):
    check_trajectory(oracle_lib, protein_small, 160, proposal=1, muex_kcal=1)


def test_runGCMC_dropin_matches_engine(protein_small):
    """gpu.runGCMC (drop-in for gcmc.gpu.runGCMC) == an Engine run of mcsteps steps."""
    from pygcmc_b200.gpu import runGCMC
    s = protein_small.copy()
    n = int(s.SimInfo[0]["mcsteps"])
    assert runGCMC(*s.arrays()) is None
    _, _, final, _ = engine_trajectory(protein_small, n)
    assert (s.fragmentInfo["totalNum"] == final.fragmentInfo["totalNum"]).all()
    a = occupied_atoms(s)
    assert np.array_equal(s.atomInfo["position"][a], final.atomInfo["position"][a])


def test_runGCMC_writes_back_what_a_full_download_holds(protein_small):
    """The drop-in copies back only what a run can change (the counts, the
    fragment residues' centres, the fragment slots' atoms); the caller's arrays
    then equal the engine's full download field for field, for ordinary and
    for page-locked host arrays."""
    from pygcmc_b200.gpu import runGCMC
    n = int(protein_small.SimInfo[0]["mcsteps"])
    _, _, final, _ = engine_trajectory(protein_small, n)
    for s in (protein_small.copy(), protein_small.pinned()):
        runGCMC(*s.arrays())
        assert np.array_equal(s.fragmentInfo, final.fragmentInfo)
        assert np.array_equal(s.residueInfo, final.residueInfo)
        assert np.array_equal(s.atomInfo, final.atomInfo)


def test_replicas_in_one_context_match_single(protein_small, water_small):
    """Several replicas advanced together give each replica's solo result."""
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    systems = [protein_small.copy(), water_small.copy(), protein_small.copy()]
    n = 100
    with Engine([x.copy() for x in systems], default_options()) as eng:
        eng.run(n)
        eng.sync()
        finals = [eng.download(r) for r in range(3)]
    for r, s in enumerate(systems):
        solo = Engine(s.copy(), default_options(replica=r))
        solo.run(n)
        solo.sync()
        f1 = solo.download()
        solo.close()
        assert (f1.fragmentInfo["totalNum"] == finals[r].fragmentInfo["totalNum"]).all()
        a = occupied_atoms(f1)
        assert np.array_equal(f1.atomInfo["position"][a], finals[r].atomInfo["position"][a])


def test_neighbour_matrix_blocks_equal_rows(protein_small):
    """Eight replicas in one context give a pose-energy launch with more items
    than resident warps, which fills the pose-pose bit matrix from mirrored
    32 x 32 blocks; each replica alone fills it row by row.  With the same
    options (the same ranges per pose) every replica's chain must be
    bit-identical to its solo run."""
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    n, nrep = 60, 8
    with Engine([protein_small.copy() for _ in range(nrep)], default_options()) as eng:
        eng.run(n)
        eng.sync()
        finals = [eng.download(r) for r in range(nrep)]
    for r in (0, 5):
        with Engine(protein_small.copy(), default_options(replica=r)) as solo:
            solo.run(n)
            solo.sync()
            f1 = solo.download()
        assert (f1.fragmentInfo["totalNum"] == finals[r].fragmentInfo["totalNum"]).all()
        a = occupied_atoms(f1)
        assert np.array_equal(f1.atomInfo["position"][a], finals[r].atomInfo["position"][a])


def test_run_in_chunks_equals_one_run(protein_small):
    from pygcmc_b200.engine import Engine
    with Engine(protein_small.copy()) as e1:
        e1.run(150)
        e1.sync()
        f1 = e1.download()
    with Engine(protein_small.copy()) as e2:
        for n in (7, 33, 1, 64, 45):
            e2.run(n)
        e2.sync()
        f2 = e2.download()
    assert (f1.fragmentInfo["totalNum"] == f2.fragmentInfo["totalNum"]).all()
    a = occupied_atoms(f1)
    assert np.array_equal(f1.atomInfo["position"][a], f2.atomInfo["position"][a])


def test_runGCMC_consecutive_calls_reuse_context(protein_small, water_small):
    """runGCMC keeps its device context between calls; a refill with a different
    system (other sizes) must give the same result as a fresh engine."""
    from pygcmc_b200._native import lib
    from pygcmc_b200.gpu import runGCMC
    for sysm in (water_small, protein_small, water_small, protein_small):
        s = sysm.copy()
        n = int(s.SimInfo[0]["mcsteps"])
        runGCMC(*s.arrays())
        _, _, final, _ = engine_trajectory(sysm, n)
        assert (s.fragmentInfo["totalNum"] == final.fragmentInfo["totalNum"]).all()
        a = occupied_atoms(s)
        assert np.array_equal(s.atomInfo["position"][a], final.atomInfo["position"][a])
    assert lib().gcmc_release_cache() == 0


def _solo_final(s, n, replica):
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    with Engine(s.copy(), default_options(replica=replica)) as e:
        e.run(n)
        e.sync()
        return e.download()


@pytest.mark.parametrize("branches,ebps", [(2, 0), (3, 1), (4, 2)])
def test_graph_branches_match_single(protein_small, water_small, branches, ebps):
    """Replicas split over concurrent graph branches (and a reduced pose-energy
    grid) give each replica's solo result."""
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    systems = [protein_small.copy(), water_small.copy(), water_small.copy(), protein_small.copy(),
               water_small.copy()]
    n = 96
    with Engine([x.copy() for x in systems], default_options(branches=branches, energy_blocks_per_sm=ebps)) as eng:
        for k in (40, 56):
            eng.run(k)
        eng.sync()
        finals = [eng.download(r) for r in range(len(systems))]
    for r, s in enumerate(systems):
        f1 = _solo_final(s, n, r)
        assert (f1.fragmentInfo["totalNum"] == finals[r].fragmentInfo["totalNum"]).all()
        a = occupied_atoms(f1)
        assert np.array_equal(f1.atomInfo["position"][a], finals[r].atomInfo["position"][a])


def test_runGCMC_batch_matches_runGCMC(protein_small, water_small):
    """The batched drop-in advances each replica exactly as its own runGCMC call
    (replica r on RNG stream r), and keeps its context between calls."""
    from pygcmc_b200._native import default_options, lib
    from pygcmc_b200.gpu import runGCMC, runGCMC_batch
    for order in ((protein_small, water_small, water_small), (water_small, protein_small, protein_small)):
        batch = [x.copy() for x in order]
        for i, b in enumerate(batch):
            b.SimInfo[0]["mcsteps"] = 60 + 20 * i
            b.SimInfo[0]["seed"] = 1000 + i
        runGCMC_batch(batch, default_options(branches=2))
        for r, src in enumerate(order):
            s = src.copy()
            s.SimInfo[0]["mcsteps"] = 60 + 20 * r
            s.SimInfo[0]["seed"] = 1000 + r
            runGCMC(*s.arrays(), options=default_options(replica=r))
            assert (s.fragmentInfo["totalNum"] == batch[r].fragmentInfo["totalNum"]).all()
            assert np.array_equal(s.atomInfo, batch[r].atomInfo)
            assert np.array_equal(s.residueInfo, batch[r].residueInfo)
    assert lib().gcmc_release_cache() == 0


def test_autotune_picks_the_fastest_trial(protein_small, water_small):
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine, autotune
    systems = [protein_small.copy(), water_small.copy(), protein_small.copy()]
    before = [s.copy() for s in systems]
    best, trials = autotune(systems, default_options(), trial_steps=32)
    assert len(trials) >= 8
    ms = [t[5] for t in trials]
    assert all(np.isfinite(ms)) and min(ms) > 0
    k = int(np.argmin(ms))
    assert (best.cells_per_cutoff, best.split_items, best.branches, best.energy_blocks_per_sm,
            best.energy_variant) == trials[k][:5]
    for s, b in zip(systems, before):  # inputs untouched
        assert np.array_equal(s.atomInfo, b.atomInfo)
        assert (s.fragmentInfo["totalNum"] == b.fragmentInfo["totalNum"]).all()
    # the tuned shape runs the same chain (check one replica against its solo run)
    with Engine([x.copy() for x in systems], best) as eng:
        eng.run(64)
        eng.sync()
        f = eng.download(1)
    solo = _solo_final(systems[1], 64, 1)
    assert (solo.fragmentInfo["totalNum"] == f.fragmentInfo["totalNum"]).all()


@pytest.mark.parametrize("proposal", [0, 2])
def test_checkpoint_resume_continues_the_chain(protein_small, proposal):
    """A context created from a checkpoint (state + remaining moves, RNG step
    offset) continues the same chain as an uninterrupted run, bit for bit."""
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    n, cut = 200, 120
    with Engine(protein_small.copy(), default_options(proposal=proposal)) as e:
        e.run(n)
        e.sync()
        full = e.download()
    with Engine(protein_small.copy(), default_options(proposal=proposal)) as e:
        e.run(cut)
        e.sync()
        ck = e.checkpoint()
    assert ck.meta["step_offset"] == cut and len(ck.moveArray) == int(protein_small.SimInfo[0]["mcsteps"]) - cut
    with Engine(ck, default_options(proposal=proposal, step_offset=ck.meta["step_offset"])) as e:
        e.run(n - cut)
        e.sync()
        res = e.download()
    assert (full.fragmentInfo["totalNum"] == res.fragmentInfo["totalNum"]).all()
    a = occupied_atoms(full)
    assert np.array_equal(full.atomInfo["position"][a], res.atomInfo["position"][a])
    r = occupied_res(full)
    assert np.array_equal(full.residueInfo["position"][r], res.residueInfo["position"][r])


def test_pair_counter_equals_oracle_pairs(oracle_lib, protein_small):
    """The engine's pair counter is the number of atom x site pairs of the
    included groups -- the oracle's count for the same insertion poses."""
    from pygcmc_b200.engine import Engine
    s = protein_small
    checked = 0
    with Engine(s.copy()) as e:
        for step in range(60):
            before = e.download()
            c0 = e.counters()["pairs"]
            e.run(1)
            e.sync()
            dp = e.counters()["pairs"] - c0
            f, m = divmod(int(s.moveArray[step]), 4)
            fr = before.fragmentInfo[f]
            if m != 0 or fr["totalNum"] >= fr["maxNum"]:
                continue
            k = int(fr["confBias"])
            ns = int(fr["num_atoms"])
            poses = [oracle_lib.insert_pose(before, f, step, i) for i in range(k)]
            xyz = np.stack([p[0] for p in poses])
            cen = np.stack([p[1] for p in poses])
            _, _, pairs = oracle_lib.energy_batch(before, xyz, fr["atoms"]["charge"][:ns],
                                                  fr["atoms"]["type"][:ns].astype(np.int32), cen, mode=0)
            assert dp == pairs, (step, dp, pairs)
            checked += 1
            if checked == 3:
                break
    assert checked >= 1


@pytest.mark.parametrize("kernel,tile_cells,cells,pair_delta", [(0, 0, 2, 0), (1, 1, 2, 0), (1, 3, 2, 0), (1, 0, 1, 0),
                                                                (1, 0, 3, 0), (0, 0, 2, -1), (1, 0, 2, -1)])
def test_trajectory_pose_energy_kernels(oracle_lib, protein_small, kernel, tile_cells, cells, pair_delta):
    """Every pose-energy kernel and launch shape replays on the oracle: the
    per-pose-warp kernel (energy_kernel 0) and the tiled kernel (1) with pose
    blocks of 1 and 3 cells and cell grids of 1 and 3 cells per cutoff;
    translate / rotate changes in the pairwise-difference form (pair_delta 0)
    and as the difference of two evaluations (-1)."""
    check_trajectory(oracle_lib, protein_small, 96, energy_kernel=kernel, tile_cells=tile_cells,
                     cells_per_cutoff=cells, pair_delta=pair_delta)


@pytest.mark.parametrize("kernel,tile_cells", [(1, 1), (0, 0)])
def test_trajectory_water_pair_image(oracle_lib, water_small, kernel, tile_cells):
    """The small water box takes the per-pair minimum image: the tiled kernel
    with one-cell pose blocks (more tiles than the default for a small box) and
    the per-pose-warp kernel, translate / rotate changes in the difference form."""
    check_trajectory(oracle_lib, water_small, 96, energy_kernel=kernel, tile_cells=tile_cells)


@pytest.mark.parametrize("which,proposal", [("protein_small", 0), ("water_small", 1)])
def test_trajectory_proportional_pose_split(request, oracle_lib, which, proposal):
    """The per-pose ranges in proportion to each pose's estimated window work
    (pose_split 1): the trajectory replays on the oracle as with uniform ranges."""
    check_trajectory(oracle_lib, request.getfixturevalue(which), 96, proposal=proposal, pose_split=1)
