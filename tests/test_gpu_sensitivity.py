"""Occupancy sensitivities (needs a B200): the configuration gradient dU/dtheta
that feeds the covariance estimator, against central finite differences of the
oracle's FP64 energies of the same configuration (1e-5 relative steps for the
LJ parameters; see below for the charges)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def frag_energy64(oracle_lib, state, ff64, charges):
    """U of the fragments: sum_f E_f(fixed) + (sum_f E_f(all) - sum_f E_f(fixed)) / 2 (FP64)."""
    from pygcmc_b200.sensitivity import _occupied
    s_all = state.copy()
    for t, f in enumerate(s_all.fragmentInfo):  # the environment carries the same charges
        ns, n, s0 = int(f["num_atoms"]), int(f["totalNum"]), int(f["startRes"])
        for j in range(n):
            a0 = int(s_all.residueInfo[s0 + j]["atomStart"])
            s_all.atomInfo["charge"][a0:a0 + ns] = charges[t]
    s_fix = s_all.copy()
    s_fix.fragmentInfo["totalNum"] = 0
    u_all = u_fix = 0.0
    for t, (xyz, cen, self_res) in enumerate(_occupied(state)):
        if len(xyz) == 0:
            continue
        f = state.fragmentInfo[t]
        ns = int(f["num_atoms"])
        ty = f["atoms"]["type"][:ns].astype(np.int32)
        u_all += oracle_lib.energy_batch64(s_all, xyz.astype(np.float64), charges[t], ty, cen, ff=ff64,
                                           self_res=self_res)[0].sum()
        u_fix += oracle_lib.energy_batch64(s_fix, xyz.astype(np.float64), charges[t], ty, cen, ff=ff64)[0].sum()
    return u_fix + 0.5 * (u_all - u_fix)


def test_configuration_gradient_matches_finite_differences(oracle_lib, protein_small):
    import torch
    from pygcmc_b200.engine import Engine
    from pygcmc_b200.grad import lj_table
    from pygcmc_b200.sensitivity import configuration_gradient
    s = protein_small
    lt = s.meta["lj_types"]
    eps, rmin = lt["eps_kcal"].astype(np.float64), lt["rmin_half"].astype(np.float64)
    ffx = int(s.SimInfo[0]["ffXNum"])
    with Engine(s.copy()) as eng:
        eng.run(40)
        eng.sync()
        state = eng.download()
        ge, gr, gq = configuration_gradient(eng, state, eps, rmin)
    charges = [f["atoms"]["charge"][: int(f["num_atoms"])].astype(np.float64) for f in state.fragmentInfo]

    def U(e, r, q):
        return frag_energy64(oracle_lib, state, lj_table(torch.tensor(e), torch.tensor(r), ffx).numpy(), q)

    checked = 0
    for which, base, g in (("eps", eps, ge), ("rmin", rmin, gr)):
        for i in np.argsort(-np.abs(g))[:3]:
            h = 1e-5 * abs(base[i])
            bp, bm = base.copy(), base.copy()
            bp[i] += h
            bm[i] -= h
            up = U(bp, rmin, charges) if which == "eps" else U(eps, bp, charges)
            um = U(bm, rmin, charges) if which == "eps" else U(eps, bm, charges)
            fd = (up - um) / (2 * h)
            assert abs(fd - g[i]) <= 2e-4 * abs(fd) + 1e-3, (which, i, fd, g[i])
            checked += 1
    # U is quadratic in the site charges, so a central difference is exact up to
    # rounding; the environment's copies of the charges are float32 (the atom
    # array), so the step must be far above their resolution: 1e-2 relative
    t = int(np.argmax(state.fragmentInfo["totalNum"]))
    for si in range(min(3, len(charges[t]))):
        h = 1e-2 * max(abs(charges[t][si]), 1e-3)
        qp = [c.copy() for c in charges]
        qm = [c.copy() for c in charges]
        qp[t][si] += h
        qm[t][si] -= h
        fd = (U(eps, rmin, qp) - U(eps, rmin, qm)) / (2 * h)
        assert abs(fd - gq[t][si]) <= 2e-4 * abs(fd) + 1e-2, (t, si, fd, gq[t][si])
        checked += 1
    assert checked == 9


def test_occupancy_sensitivity_runs(protein_small):
    from pygcmc_b200._native import default_options
    from pygcmc_b200.sensitivity import occupancy_sensitivity
    lt = protein_small.meta["lj_types"]
    r = occupancy_sensitivity(protein_small, default_options(), nsamples=6, stride=20,
                              eps_kcal=lt["eps_kcal"], rmin_half=lt["rmin_half"])
    nt = len(protein_small.fragmentInfo)
    assert r["dN_deps"].shape == (nt, len(lt["eps_kcal"])) and np.isfinite(r["dN_deps"]).all()
    assert r["dN_dq"].shape[0] == nt and np.isfinite(r["dN_dq"]).all()
