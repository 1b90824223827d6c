"""The persistent step loop (gcmc_options.persistent = 1): one cooperative
launch runs a batched context's steps with grid barriers between the
pose-energy and the accept phases, in place of the captured graph of per-step
launches (needs a B200).

* Every replica's chain -- per-step logs, logged pose energies, counters and
  the final state -- is bit-identical to the graph's (the same items and the
  same summation order; only which warp takes an item differs).
* Runs in several calls continue one chain.
* A barrier wait cap of one poll makes the CTAs give up at the first barrier:
  the launch ends, the device error word carries bit 5 and the host reports
  it, with no fault (the context is then discarded).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LOG_KMAX = 1024


def _run(systems, nsteps, chunks=None, **opt):
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    opts = default_options(log_steps=nsteps, log_kmax=LOG_KMAX, **opt)
    with Engine([s.copy() for s in systems], opts) as eng:
        for n in (chunks or [nsteps]):
            eng.run(n)
        eng.sync()
        assert eng.device_error() == 0
        out = []
        for r in range(len(systems)):
            logs, E = eng.logs(r)
            out.append((logs, E, eng.download(r), eng.counters(r)))
    return out


def _same(a, b):
    for (la, Ea, fa, ca), (lb, Eb, fb, cb) in zip(a, b):
        for f in la.dtype.names:
            assert np.array_equal(la[f], lb[f]), f
        assert np.array_equal(Ea.view(np.uint64), Eb.view(np.uint64))
        assert ca == cb
        assert np.array_equal(fa.fragmentInfo["totalNum"], fb.fragmentInfo["totalNum"])
        assert np.array_equal(fa.atomInfo["position"], fb.atomInfo["position"])
        assert np.array_equal(fa.residueInfo["position"], fb.residueInfo["position"])


@pytest.fixture(scope="module")
def batch(protein_small, water_small):
    return [protein_small, water_small, protein_small, water_small, protein_small]


def test_persistent_equals_graph(batch):
    n = 80
    graph = _run(batch, n)
    pers = _run(batch, n, persistent=1)
    _same(graph, pers)
    assert any((lg["n_accept"] > 0).any() for lg, _, _, _ in pers)


def test_persistent_in_chunks(batch):
    n = 75
    _same(_run(batch, n, persistent=1), _run(batch, n, chunks=[30, 1, 44], persistent=1))


def test_persistent_barrier_cap_ends_the_launch(batch):
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    eng = Engine([s.copy() for s in batch], default_options(persistent=1, persist_spin_cap=1))
    try:
        eng.run(20)
        with pytest.raises(RuntimeError):
            eng.sync()
        assert eng.device_error() & 32
    finally:
        eng.close()
