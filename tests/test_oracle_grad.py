"""The oracle's FP64 analytic gradients of the pose energy against central
finite differences of its FP64 energies (no GPU).  Steps: 1e-4 A on site
coordinates, 1e-5 relative on site charges and pair-table entries.

Random poses (uniform centre in the box) include deep clashes whose energies
reach 1e12 kJ/mol; a central difference of such energies is dominated by
their rounding, so the finite-difference checks use the poses whose sum of
|pair terms| is below 1e8 kJ/mol (the analytic gradients of all poses are
checked against the GPU elsewhere)."""
import numpy as np
import pytest

from pygcmc_b200 import poses as PZ


@pytest.fixture(scope="module")
def case(protein_small):
    s = protein_small
    tpl, q, t = PZ.template(s, 2)
    com, quat = PZ.random_poses(s, 96, seed=5)
    xyz = PZ.rigid_sites(tpl, com, quat)
    return s, xyz, q.astype(np.float64), t, com.astype(np.float32)


def well_conditioned(oracle_lib, case):
    s, xyz, q, t, cen = case
    _, _, _, El1 = oracle_lib.energy_batch(s, xyz.astype(np.float32), q.astype(np.float32), t, cen, mode=0,
                                           want_l1=True)
    ok = El1 < 1e8
    assert ok.sum() >= 16
    return s, xyz[ok], q, t, cen[ok]


def test_site_gradient_matches_finite_differences(oracle_lib, case):
    s, xyz, q, t, cen = well_conditioned(oracle_lib, case)
    g = oracle_lib.grad_batch(s, xyz, q, t, cen)
    E0, ng0 = oracle_lib.energy_batch64(s, xyz, q, t, cen)
    assert (ng0 > 0).sum() > 10
    # l1 scale of each pose energy: the rounding of E(x +- h) is ~eps * El1
    _, _, _, El1 = oracle_lib.energy_batch(s, xyz.astype(np.float32), q.astype(np.float32), t, cen, mode=0,
                                           want_l1=True)
    h = 1e-4
    ns = xyz.shape[1]
    worst = 0.0
    for si in range(ns):
        for c in range(3):
            xp, xm = xyz.copy(), xyz.copy()
            xp[:, si, c] += h
            xm[:, si, c] -= h
            fd = (oracle_lib.energy_batch64(s, xp, q, t, cen)[0] - oracle_lib.energy_batch64(s, xm, q, t, cen)[0]) / (2 * h)
            # central-difference truncation O(h^2) plus the rounding of the two energies
            tol = 1e-5 * g["gxyz_l1"][:, si] + 64 * 2.2e-16 * El1 / (2 * h)
            err = np.abs(fd - g["gxyz"][:, si, c]) / tol
            worst = max(worst, float(err.max()))
    assert worst <= 1.0, worst


def test_charge_gradient_matches_finite_differences(oracle_lib, case):
    s, xyz, q, t, cen = well_conditioned(oracle_lib, case)
    g = oracle_lib.grad_batch(s, xyz, q, t, cen)
    _, _, _, El1 = oracle_lib.energy_batch(s, xyz.astype(np.float32), q.astype(np.float32), t, cen, mode=0,
                                           want_l1=True)
    for si in range(len(q)):
        h = 1e-5 * abs(q[si])
        qp, qm = q.copy(), q.copy()
        qp[si] += h
        qm[si] -= h
        fd = (oracle_lib.energy_batch64(s, xyz, qp, t, cen)[0] - oracle_lib.energy_batch64(s, xyz, qm, t, cen)[0]) / (2 * h)
        # the energy is linear in q: the difference is exact up to the rounding of the energies
        tol = 1e-9 * g["gq_l1"][:, si] + 64 * 2.2e-16 * El1 / (2 * h)
        assert np.all(np.abs(fd - g["gq"][:, si]) <= tol), si


def test_table_gradient_matches_finite_differences(oracle_lib, case):
    s, xyz, q, t, cen = well_conditioned(oracle_lib, case)
    rng = np.random.default_rng(2)
    gout = rng.normal(size=len(xyz))
    g = oracle_lib.grad_batch(s, xyz, q, t, cen, gout=gout)
    _, _, _, El1 = oracle_lib.energy_batch(s, xyz.astype(np.float32), q.astype(np.float32), t, cen, mode=0,
                                           want_l1=True)
    ff = s.ff.astype(np.float64)
    used = np.flatnonzero(g["gff_l1"] > 0)
    assert len(used) > 10
    for j in rng.choice(used, 12, replace=False):
        h = 1e-5 * abs(ff[j])
        fp, fm = ff.copy(), ff.copy()
        fp[j] += h
        fm[j] -= h
        Lp = gout @ oracle_lib.energy_batch64(s, xyz, q, t, cen, ff=fp)[0]
        Lm = gout @ oracle_lib.energy_batch64(s, xyz, q, t, cen, ff=fm)[0]
        fd = (Lp - Lm) / (2 * h)
        tol = 1e-5 * g["gff_l1"][j] + 64 * 2.2e-16 * (np.abs(gout) @ El1) / (2 * h)
        assert abs(fd - g["gff"][j]) <= tol, (j, fd, g["gff"][j], g["gff_l1"][j])


def test_fp64_energy_agrees_with_float_input_energy(oracle_lib, case):
    s, xyz, q, t, cen = case
    x32 = xyz.astype(np.float32)
    e64, ng64 = oracle_lib.energy_batch64(s, x32.astype(np.float64), q.astype(np.float32).astype(np.float64), t, cen,
                                          ff=s.ff.astype(np.float64))
    e, ng, _ = oracle_lib.energy_batch(s, x32, q.astype(np.float32), t, cen, mode=0)
    assert np.array_equal(ng, ng64)
    assert np.allclose(e, e64, rtol=1e-12, atol=1e-9)
