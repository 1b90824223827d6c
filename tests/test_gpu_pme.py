"""Smooth-PME electrostatics against the oracle's exact Ewald sums (needs a B200).

* the mesh potential converges to the exact Ewald reciprocal potential as the
  mesh is refined (order-4 B-splines), below 1e-4 of its RMS on a 0.4 A mesh;
* trajectories with Ewald electrostatics replay on the oracle with identical
  decisions and running energies; each trial energy is within
  1e-5 of its sum of |terms| plus the PME discretisation error of its sites'
  potentials (4x the largest |phi_PME - phi_Ewald| seen at random points of
  the starting state, times sum |q_s|, twice for translate/rotate);
* the same with force-biased translate/rotate moves: the oracle replays the
  engine's energies and forces (identical decisions and final coordinates),
  and the engine's forces and torques (real-space erfc pairs, the mesh
  potential's gradient, the molecular term) lie within the mesh's
  discretisation error of the oracle's exact-Ewald FP64 values.
"""
import numpy as np
import pytest

from test_gpu_parity import LOG_FIELDS, LOG_KMAX, occupied_atoms

pytestmark = pytest.mark.gpu

ALPHA = 0.32


def pme_options(grid, **kw):
    from pygcmc_b200._native import default_options
    o = default_options(pme=1, pme_alpha=ALPHA, **kw)
    for a in range(3):
        o.pme_grid[a] = grid
    return o


def phi_error(oracle_lib, system, grid, npts=400):
    from pygcmc_b200.engine import Engine
    L = system.SimInfo[0]["cryst"].astype(float)
    st = system.SimInfo[0]["startxyz"].astype(float)
    pts = st + np.random.default_rng(7).random((npts, 3)) * L
    ref = oracle_lib.ewald_potential(system, ALPHA, pts)
    with Engine(system.copy(), pme_options(grid)) as e:
        phi = e.pme_potential(pts)
    return float(np.abs(phi - ref).max()), float(np.sqrt((ref ** 2).mean()))


def test_pme_potential_converges_to_ewald(oracle_lib, water_small):
    errs = []
    for grid in (16, 32, 64):
        err, rms = phi_error(oracle_lib, water_small, grid)
        errs.append(err)
        print(f"mesh {grid}^3: max |phi_pme - phi_ewald| = {err:.3e} (rms phi {rms:.1f})")
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] <= 1e-4 * rms


@pytest.mark.parametrize("which,nsteps", [("water_small", 40), ("protein_small", 24)])
def test_pme_trajectory_replays_on_oracle(request, oracle_lib, which, nsteps):
    from pygcmc_b200.engine import Engine
    system = request.getfixturevalue(which)
    grid = 64
    dphi, _ = phi_error(oracle_lib, system, grid)
    with Engine(system.copy(), pme_options(grid, log_steps=nsteps, log_kmax=LOG_KMAX)) as e:
        e.run(nsteps)
        e.sync()
        logs_g, E_g = e.logs()
        final_g = e.download()
    s_o = system.copy()
    r = oracle_lib.run_ext(s_o, nsteps, opts=oracle_lib.options(pme=1, pme_alpha=ALPHA), kmax=LOG_KMAX, replay=E_g)
    logs_o = r["logs"]
    for f in LOG_FIELDS:
        assert np.array_equal(logs_g[f], logs_o[f]), f
    assert np.array_equal(logs_g["e_total"], logs_o["e_total"])
    qabs = np.array([np.abs(fr["atoms"]["charge"][: int(fr["num_atoms"])]).sum() for fr in system.fragmentInfo])
    mask = np.arange(LOG_KMAX)[None, :] < logs_g["k"][:, None]
    mult = np.where(np.isin(logs_g["move"], [2, 3]), 2.0, 1.0) * qabs[logs_g["ftype"]]
    tol = 1e-5 * r["scale"] + 4.0 * dphi * mult[:, None]
    bad = mask & ~(np.abs(E_g - r["energies"]) <= tol)
    assert not bad.any(), (np.argwhere(bad)[:5], E_g[bad][:5], r["energies"][bad][:5], tol[bad][:5])
    a = occupied_atoms(s_o)
    assert np.array_equal(final_g.atomInfo["position"][a], s_o.atomInfo["position"][a])
    print(f"{which}: PME max |phi err| {dphi:.2e}; trn/rot/ins/del energies within bound")


def test_pme_replicas_match_single(protein_small, water_small):
    from pygcmc_b200.engine import Engine
    systems = [water_small.copy(), protein_small.copy()]
    n = 40
    with Engine([x.copy() for x in systems], pme_options(32, branches=2)) as e:
        e.run(n)
        e.sync()
        finals = [e.download(k) for k in range(2)]
    for k, s in enumerate(systems):
        o = pme_options(32)
        o.replica = k
        with Engine(s.copy(), o) as e1:
            e1.run(n)
            e1.sync()
            f1 = e1.download()
        a = occupied_atoms(f1)
        assert (f1.fragmentInfo["totalNum"] == finals[k].fragmentInfo["totalNum"]).all()
        assert np.array_equal(f1.atomInfo["position"][a], finals[k].atomInfo["position"][a])


def test_pme_dropin_repeated_calls_match_engine(water_small):
    """Drop-in calls with Ewald electrostatics: the second call refills the
    context kept from the first (its mesh buffers and influence function are
    reused); both give the result of a fresh engine run of the same steps."""
    from pygcmc_b200.engine import Engine
    from pygcmc_b200.gpu import runGCMC
    n = 40
    base = water_small.copy()
    base.SimInfo[0]["mcsteps"] = n
    base.moveArray = np.ascontiguousarray(base.moveArray[:n])
    with Engine(base.copy(), pme_options(32)) as e:
        e.run(n)
        e.sync()
        final = e.download()
    for _ in range(2):
        s = base.copy()
        runGCMC(*s.arrays(), options=pme_options(32))
        assert (s.fragmentInfo["totalNum"] == final.fragmentInfo["totalNum"]).all()
        a = occupied_atoms(s)
        assert np.array_equal(s.atomInfo["position"][a], final.atomInfo["position"][a])


def test_pme_force_biased_trajectory_replays_on_oracle(oracle_lib, water_small):
    from pygcmc_b200.engine import Engine
    nsteps, grid = 48, 64
    opts = pme_options(grid, proposal=2, log_steps=nsteps, log_kmax=LOG_KMAX)
    with Engine(water_small.copy(), opts) as e:
        e.run(nsteps)
        e.sync()
        logs_g, E_g = e.logs()
        F_g = e.forces()
        final_g = e.download()
    s_o = water_small.copy()
    oo = oracle_lib.options(proposal=2, pme=1, pme_alpha=ALPHA, fb_trn=float(opts.fb_trn), fb_rot=float(opts.fb_rot))
    r = oracle_lib.run_ext(s_o, nsteps, opts=oo, kmax=LOG_KMAX, replay=E_g, replay_forces=F_g)
    logs_o = r["logs"]
    for f in LOG_FIELDS:
        assert np.array_equal(logs_g[f], logs_o[f]), f
    assert np.array_equal(logs_g["e_total"], logs_o["e_total"])
    a = occupied_atoms(s_o)
    assert np.array_equal(final_g.atomInfo["position"][a], s_o.atomInfo["position"][a])
    mask = np.arange(LOG_KMAX)[None, :] < logs_g["k"][:, None]
    fbm = mask & np.isin(logs_g["move"], [2, 3])[:, None]
    assert fbm.sum() > 20
    Fg = F_g[fbm].astype(np.float64)
    Fo = r["forces"][fbm]
    sc = np.repeat(r["fscale"][fbm], 3, axis=1)
    fin = np.isfinite(Fg) & (sc < 1e30)
    rel = np.abs(Fg - Fo)[fin] / np.maximum(sc[fin], 1e-30)
    print(f"PME force-biased: max |force err| / l1 = {rel.max():.2e}, median {np.median(rel):.2e}; "
          f"trn/rot accepted {logs_g['n_accept'][np.isin(logs_g['move'], [2, 3])].sum()}")
    # the mesh gradient's discretisation error on a 0.4 A mesh: well below 1e-3 of the l1 scale
    assert rel.max() < 1e-3

