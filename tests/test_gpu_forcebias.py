"""Force-biased translate/rotate moves (proposal 2) against the oracle (needs a B200).

The oracle replays the engine's logged pose energies and forces: every step's
decisions and counts must be identical, the running energy bit-identical, the
final coordinates bit-identical (the proposal is a deterministic function of
the force floats and the counter-based RNG), and the engine's forces and
torques within 1e-5 of the l1 scale of their pair terms of the oracle's FP64
values (1e-4 relative to the pose energy's l1 where forces overflow FP32 on
deep clashes is not reached by the test systems).
"""
import numpy as np
import pytest

from conftest import energy_close
from test_gpu_parity import LOG_FIELDS, LOG_KMAX, occupied_atoms, occupied_res

pytestmark = pytest.mark.gpu

FORCE_REL = 1e-5


def fb_trajectory(oracle, system, nsteps, **kw):
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    opts = default_options(log_steps=nsteps, log_kmax=LOG_KMAX, proposal=2, **kw)
    with Engine(system.copy(), opts) as eng:
        for n in (nsteps // 3, nsteps - nsteps // 3):
            eng.run(n)
        eng.sync()
        logs_g, E_g = eng.logs()
        F_g = eng.forces()
        final_g = eng.download()
        et = eng.energy_total()
    s_o = system.copy()
    oo = oracle.options(proposal=2, fb_trn=float(opts.fb_trn), fb_rot=float(opts.fb_rot))
    r = oracle.run_ext(s_o, nsteps, opts=oo, kmax=LOG_KMAX, replay=E_g, replay_forces=F_g)
    return logs_g, E_g, F_g, final_g, et, s_o, r


@pytest.mark.parametrize("which", ["protein_small", "water_small"])
def test_force_biased_trajectory_matches_oracle(request, oracle_lib, which):
    system = request.getfixturevalue(which)
    nsteps = 160
    logs_g, E_g, F_g, final_g, et, s_o, r = fb_trajectory(oracle_lib, system, nsteps)
    logs_o = r["logs"]
    for f in LOG_FIELDS:
        bad = np.flatnonzero(logs_g[f] != logs_o[f])
        assert bad.size == 0, (f, bad[:5], logs_g[bad[:3]], logs_o[bad[:3]])
    assert np.array_equal(logs_g["e_total"], logs_o["e_total"])
    assert et == logs_g["e_total"][-1]
    mask = np.arange(LOG_KMAX)[None, :] < logs_g["k"][:, None]
    assert energy_close(E_g[mask], r["energies"][mask], r["scale"][mask]).all()
    # forces and torques of the force-biased poses
    fbm = mask & np.isin(logs_g["move"], [2, 3])[:, None]
    assert fbm.sum() > 50
    Fg = F_g[fbm].astype(np.float64)            # [n, 12]
    Fo = r["forces"][fbm]                       # [n, 12]
    sc = r["fscale"][fbm]                       # [n, 4]: F_old, tau_old, F_new, tau_new
    scale = np.repeat(sc, 3, axis=1)            # per component
    fin = np.isfinite(Fg) & (scale < 1e30)
    tol = FORCE_REL * scale + 1e-5
    bad = fin & ~(np.abs(Fg - Fo) <= tol)
    assert not bad.any(), (np.argwhere(bad)[:5], Fg[bad][:5], Fo[bad][:5], scale[bad][:5])
    err = np.abs(Fg - Fo)[fin] / np.maximum(scale[fin], 1e-30)
    print(f"{which}: max |force err| / l1 = {err.max():.2e}; "
          f"trn/rot acceptance {logs_g['n_accept'][np.isin(logs_g['move'], [2, 3])].sum()} "
          f"of {logs_g['k'][np.isin(logs_g['move'], [2, 3])].sum()} poses")
    assert (final_g.fragmentInfo["totalNum"] == s_o.fragmentInfo["totalNum"]).all()
    a = occupied_atoms(s_o)
    assert np.array_equal(final_g.atomInfo["position"][a], s_o.atomInfo["position"][a])
    rr = occupied_res(s_o)
    assert np.array_equal(final_g.residueInfo["position"][rr], s_o.residueInfo["position"][rr])


@pytest.mark.parametrize("branches", [1, 2])
def test_force_biased_replicas_and_branches_match_single(protein_small, water_small, branches):
    """Replicas with different move schedules in one context (a launch then holds
    force-biased and plain items, split between SMs) give each replica the chain it
    has alone."""
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    systems = [protein_small.copy(), water_small.copy(), protein_small.copy()]
    n = 64
    with Engine([x.copy() for x in systems], default_options(proposal=2, branches=branches)) as eng:
        eng.run(n)
        eng.sync()
        finals = [eng.download(k) for k in range(3)]
        e_tot = [eng.energy_total(k) for k in range(3)]
    for k, s in enumerate(systems):
        with Engine(s.copy(), default_options(proposal=2, replica=k)) as e1:
            e1.run(n)
            e1.sync()
            f1 = e1.download()
            assert e1.energy_total() == e_tot[k]
        a = occupied_atoms(f1)
        assert (f1.fragmentInfo["totalNum"] == finals[k].fragmentInfo["totalNum"]).all()
        assert np.array_equal(f1.atomInfo["position"][a], finals[k].atomInfo["position"][a])
