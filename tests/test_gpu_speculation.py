"""Speculative next-step evaluation (gcmc_options.speculate) against the
sequential step order (needs a B200).

A one-replica context prepares step j + 1 and evaluates its pose energies
while step j's accept kernel runs, and keeps them when step j accepted
nothing.  Every logged field, every logged pose energy, the final state and
the pair counter must then be bit-identical to the sequential order's, on
systems whose steps accept often (water) and rarely (protein).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LOG_KMAX = 1024


def _run(system, nsteps, speculate, chunks=None, kernel=0, **kw):
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    opts = default_options(log_steps=nsteps, log_kmax=LOG_KMAX, speculate=speculate, energy_kernel=kernel, **kw)
    with Engine(system.copy(), opts) as eng:
        if chunks is None:
            eng.run(nsteps)
        else:
            for kind, n in chunks:
                if kind == "graph":
                    eng.run(n)
                else:
                    eng.run_profiled(n)
        eng.sync()
        assert eng.device_error() == 0
        logs, E = eng.logs()
        return logs, E, eng.download(), eng.counters(), eng.phase_cycles()


def _same(a, b):
    logs_a, E_a, fin_a, cnt_a, _ = a
    logs_b, E_b, fin_b, cnt_b, _ = b
    assert len(logs_a) == len(logs_b)
    for f in logs_a.dtype.names:
        bad = np.flatnonzero(logs_a[f] != logs_b[f])
        assert bad.size == 0, (f, bad[:5])
    assert np.array_equal(E_a.view(np.uint64), E_b.view(np.uint64))
    assert cnt_a == cnt_b
    assert np.array_equal(fin_a.fragmentInfo["totalNum"], fin_b.fragmentInfo["totalNum"])
    assert np.array_equal(fin_a.atomInfo["position"], fin_b.atomInfo["position"])
    assert np.array_equal(fin_a.residueInfo["position"], fin_b.residueInfo["position"])


@pytest.mark.parametrize("kernel", [0, 1], ids=["per_pose", "tiled"])
@pytest.mark.parametrize("which", ["protein_small", "water_small"])
def test_speculation_equals_sequential_order(request, which, kernel):
    s = request.getfixturevalue(which)
    n = int(s.SimInfo[0]["mcsteps"])
    on = _run(s, n, 0, kernel=kernel)
    off = _run(s, n, -1, kernel=kernel)
    _same(on, off)
    kept = int(on[4][6])
    accepted_steps = int((on[0]["n_accept"] > 0).sum())
    # a step's speculation is kept iff the step before it accepted nothing
    assert 0 < kept <= n - accepted_steps
    assert int(off[4][6]) == 0


@pytest.mark.parametrize("kernel", [0, 1], ids=["per_pose", "tiled"])
def test_speculation_on_the_benchmark_protein(kernel):
    """6000 atoms, 1000 insertion poses: the one-wave split and the mirrored
    neighbour blocks of the benchmark workload (tiled: blocks holding more
    poses than one tile, cut into several tiles)."""
    from pygcmc_b200 import system as S
    s = S.protein_system(seed=1, mcsteps=300)
    _same(_run(s, 300, 0, kernel=kernel), _run(s, 300, -1, kernel=kernel))


def test_speculation_mixed_with_timed_steps(protein_small):
    """Graph runs (speculating) interleaved with step-by-step timed runs
    (sequential, first descriptor copy) continue one chain."""
    chunks = [("graph", 37), ("timed", 5), ("graph", 60), ("timed", 3), ("graph", 21), ("graph", 1)]
    n = sum(c[1] for c in chunks)
    _same(_run(protein_small, n, 0, chunks), _run(protein_small, n, -1))


def _occupied_atoms(s):
    idx = []
    for f in s.fragmentInfo:
        for j in range(int(f["totalNum"])):
            r = s.residueInfo[int(f["startRes"]) + j]
            idx.extend(range(int(r["atomStart"]), int(r["atomStart"]) + int(r["atomNum"])))
    return np.array(idx, dtype=np.int64)


def test_dropin_refills_switching_speculation(protein_small, water_small):
    """The drop-in's kept context is refilled with speculation switched off and
    on again (per-step buffers and captured graphs change); every call equals
    a fresh engine with the same options."""
    from pygcmc_b200._native import default_options, lib
    from pygcmc_b200.gpu import runGCMC
    for sysm, spec in ((water_small, 0), (protein_small, -1), (water_small, -1), (protein_small, 0)):
        s = sysm.copy()
        n = int(s.SimInfo[0]["mcsteps"])
        runGCMC(*s.arrays(), options=default_options(speculate=spec))
        _, _, fin, _, _ = _run(sysm, n, spec)
        assert np.array_equal(s.fragmentInfo["totalNum"], fin.fragmentInfo["totalNum"])
        a = _occupied_atoms(s)
        assert np.array_equal(s.atomInfo["position"][a], fin.atomInfo["position"][a])
    assert lib().gcmc_release_cache() == 0


def test_speculation_with_proportional_pose_split(protein_small):
    """Per-pose ranges in proportion to the estimated window work (pose_split 1):
    the speculative and the sequential orders stay bit-identical."""
    n = int(protein_small.SimInfo[0]["mcsteps"])
    _same(_run(protein_small, n, 0, pose_split=1), _run(protein_small, n, -1, pose_split=1))
