"""Oracle parity on the benchmark configurations themselves (needs a B200).

Each case runs the engine with per-step logs, replays the step sequence on the
FP64 oracle with the engine's energies (so the two take the same decisions and
stay on one trajectory), and checks:

* every logged field, the running energy and the final state equal the
  oracle's (decision parity; bit-identical counts, slots and coordinates);
* the per-trial criterion: |dE_gpu - dE_oracle| <= max(1e-5 |dE_oracle|,
  1e-4 kcal/mol), dE the pose energy of an insertion / deletion or
  E_new - E_old of a translate / rotate; the fraction meeting it is printed
  and must reach REQUIRED_FRACTION; every trial must meet the looser bound
  relative to its sum of |pair terms| (the condition of the FP32 sum);
* decisions: the oracle counts the acceptance decisions whose draw lies
  within the per-trial tolerance of its threshold (the only ones two valid
  evaluations may take differently), and an oracle run on its own FP64
  energies, without replay, must take the engine's decisions at every step
  whenever that count is 0.

Cases: the benchmark protein system exactly (6000 fixed atoms, 64 A box,
8 fragments, confBias 1000, reference proposals); the water box of 800 TIP3P
waters in 30 A with symmetric 1 A-cube / 15-degree moves and muex in kcal/mol;
and both ends of the batched replicas' size range (2000 and 40000 fixed atoms,
muex scan ends), run together in one context.
"""
import numpy as np
import pytest

from conftest import ABS_TOL_KJ, REL_TOL, energy_close
from test_gpu_parity import LOG_FIELDS, LOG_KMAX, occupied_atoms, occupied_res

pytestmark = pytest.mark.gpu

# fraction of trial energies that must meet the per-trial criterion literally
REQUIRED_FRACTION = 0.999


def literal_ok(e_gpu, e_orc):
    return np.abs(e_gpu - e_orc) <= np.maximum(REL_TOL * np.abs(e_orc), ABS_TOL_KJ)


def check_replay(oracle, system, logs_g, E_g, final_g, nsteps, opts, label):
    s_o = system.copy()
    oracle.decision_stats(reset=True)
    r = oracle.run_ext(s_o, nsteps, opts=opts, kmax=LOG_KMAX, replay=E_g)
    n_dec, n_band, min_ratio = oracle.decision_stats(reset=True)
    logs_o, E_o, SC = r["logs"], r["energies"], r["scale"]
    for f in LOG_FIELDS:
        bad = np.flatnonzero(logs_g[f] != logs_o[f])
        assert bad.size == 0, (label, f, bad[:5])
    assert np.array_equal(logs_g["e_total"], logs_o["e_total"]), label
    assert np.array_equal(final_g.fragmentInfo["totalNum"], s_o.fragmentInfo["totalNum"]), label
    a = occupied_atoms(s_o)
    assert np.array_equal(final_g.atomInfo["position"][a], s_o.atomInfo["position"][a]), label
    rr = occupied_res(s_o)
    assert np.array_equal(final_g.residueInfo["position"][rr], s_o.residueInfo["position"][rr]), label
    mask = np.arange(LOG_KMAX)[None, :] < logs_g["k"][:, None]
    eg, eo, sc = E_g[mask], E_o[mask], SC[mask]
    fin = np.isfinite(eo)
    assert np.array_equal(np.isfinite(eg), fin), label
    eg, eo, sc = eg[fin], eo[fin], sc[fin]
    assert energy_close(eg, eo, sc).all(), (label, "sum-of-|terms| bound")
    lit = literal_ok(eg, eo)
    rel = np.abs(eg - eo) / np.maximum(np.abs(eo), 1e-300)
    moves = np.repeat(logs_g["move"], logs_g["k"])[fin]
    per_move = {m: float(lit[moves == m].mean()) for m in range(4) if (moves == m).any()}
    worst = np.argmax(np.abs(eg - eo) / np.maximum(REL_TOL * np.abs(eo), ABS_TOL_KJ))
    print(f"\n[{label}] {nsteps} steps, {eg.size} finite trial energies: {lit.mean() * 100:.3f}% within "
          f"1e-5 |dE| or 1e-4 kcal/mol (per move {per_move}); median rel err {np.median(rel):.2e}; worst "
          f"err/tol {np.abs(eg - eo)[worst] / max(REL_TOL * abs(eo[worst]), ABS_TOL_KJ):.2f} at dE {eo[worst]:.4g} "
          f"kJ/mol; {n_dec} decisions, {n_band} within the tolerance band of their threshold "
          f"(min margin/tol {min_ratio:.3g})")
    assert lit.mean() >= REQUIRED_FRACTION, (label, lit.mean())
    # the oracle's own FP64 energies, no replay: the same decisions unless one lies in the band
    s_f = system.copy()
    r_f = oracle.run_ext(s_f, nsteps, opts=opts, kmax=LOG_KMAX)
    same = all(np.array_equal(logs_g[f], r_f["logs"][f]) for f in LOG_FIELDS)
    print(f"[{label}] oracle on its own FP64 energies takes the engine's decisions at every step: {same}")
    if n_band == 0:
        assert same, label
    return lit.mean(), n_dec, n_band


def run_logged(systems, nsteps, **opt):
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    opts = default_options(log_steps=nsteps, log_kmax=LOG_KMAX, **opt)
    with Engine([s.copy() for s in systems], opts) as eng:
        eng.run(nsteps)
        eng.sync()
        out = []
        for r in range(len(systems)):
            logs, E = eng.logs(r)
            out.append((logs, E, eng.download(r)))
    return out


# both pose-energy kernels: one warp per pose and cell range (0) and tiled (1)
KERNELS = pytest.mark.parametrize("kernel", [0, 1], ids=["per_pose", "tiled"])


@KERNELS
def test_benchmark_protein_system(oracle_lib, kernel):
    """The bench's workload exactly: protein_system(seed=1), 6000 fixed atoms, confBias 1000."""
    from pygcmc_b200 import system as S
    n = 256
    s = S.protein_system(seed=1, mcsteps=n)
    assert int(s.meta["n_fixed"]) == 6000 and int(s.fragmentInfo[0]["confBias"]) == 1000
    (logs, E, final), = run_logged([s], n, energy_kernel=kernel)
    assert set(np.unique(logs["move"])) == {0, 1, 2, 3}
    assert (logs["n_accept"] > 0).any()
    check_replay(oracle_lib, s, logs, E, final, n, oracle_lib.options(), f"protein 6000, confBias 1000, kernel {kernel}")


@KERNELS
def test_water_box_symmetric_moves(oracle_lib, kernel):
    """800 TIP3P waters, 30 A box, muex -5.8 kcal/mol, 55 M, translate in a 1 A cube, rotate <= 15 degrees."""
    from pygcmc_b200 import system as S
    n = 256
    s = S.water_box(n_water=800, box=30.0, seed=1, mcsteps=n)
    rot = float(np.radians(15.0))
    (logs, E, final), = run_logged([s], n, proposal=1, muex_kcal=1, trn_step=1.0, rot_max=rot, energy_kernel=kernel)
    assert set(np.unique(logs["move"])) == {0, 1, 2, 3}
    check_replay(oracle_lib, s, logs, E, final, n,
                 oracle_lib.options(proposal=1, muex_kcal=1, trn_step=1.0, rot_max=rot),
                 f"water 800, 30 A, kernel {kernel}")


def test_batched_replica_size_extremes(oracle_lib):
    """Replicas at both ends of the batched range (2000 and 40000 fixed atoms, box and
    radius scaled as the batch builder scales them, muex shifted by -8 and 0), in one context."""
    import math
    from pygcmc_b200 import system as S
    n = 128
    density = 6000 / 64.0 ** 3
    systems = []
    for i, (atoms, shift) in enumerate([(2000, -8.0), (40000, 0.0)]):
        box = float(np.clip((atoms / density) ** (1.0 / 3.0), 40.0, 100.0))
        radius = min(24.0 * (atoms / 6000.0) ** (1.0 / 3.0), box / 2 - 2.0)
        systems.append(S.protein_system(seed=1000 + i, n_atoms=atoms, box=box, radius=radius, mcsteps=n,
                                        muex_shift=shift))
    assert math.isclose(float(systems[1].SimInfo[0]["cryst"][0]), 100.0)
    res = run_logged(systems, n)
    for r, (s, (logs, E, final)) in enumerate(zip(systems, res)):
        check_replay(oracle_lib, s, logs, E, final, n, oracle_lib.options(replica=r),
                     f"batched replica {r}: {int(s.meta['n_fixed'])} atoms")
