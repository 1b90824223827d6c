"""Host-side pieces of the force-biased proposal (no GPU): the own logarithm
and exponential, and a force-biased oracle run."""
import numpy as np


def test_det_log_accuracy(oracle_lib):
    L = oracle_lib.lib()
    xs = np.concatenate([np.linspace(1e-7, 1.0, 2001, dtype=np.float32),
                         np.float32(2.0) ** np.arange(-24, 1, dtype=np.float32)])
    got = np.array([L.or_det_log(float(x)) for x in xs], dtype=np.float64)
    ref = np.log(xs.astype(np.float64))
    assert np.all(np.abs(got - ref) <= 4e-7 * np.maximum(np.abs(ref), 1.0))


def test_det_exp_accuracy(oracle_lib):
    L = oracle_lib.lib()
    xs = np.concatenate([np.linspace(-86.9, 0.0, 4001, dtype=np.float32), np.float32([-1e-6, -0.3466, -0.3467])])
    got = np.array([L.or_det_exp_neg(float(x)) for x in xs], dtype=np.float64)
    ref = np.exp(xs.astype(np.float64))
    assert np.all(np.abs(got - ref) <= 4e-7 * ref)
    assert L.or_det_exp_neg(-90.0) == 0.0


def test_force_biased_oracle_run(oracle_lib, protein_small):
    s = protein_small.copy()
    r = oracle_lib.run_ext(s, 60, opts=oracle_lib.options(proposal=2), kmax=1024)
    logs = r["logs"]
    tr = np.isin(logs["move"], [2, 3])
    assert tr.sum() > 10
    assert (logs["n_accept"][tr] <= logs["k"][tr]).all() and logs["n_accept"][tr].sum() > 0
    f = r["forces"][tr][:, :1]
    assert np.isfinite(f).all()
    assert r["e_total"] == logs["e_total"][-1]
