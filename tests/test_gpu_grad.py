"""Backward kernel and autograd wrapper vs the FP64 oracle (needs a B200).

* gcmc_energy_grad's per-pose site and charge gradients and its weighted
  pair-table gradient against the oracle's FP64 analytic gradient at the same
  (float32) sites: |g_gpu - g_fp64| <= 1e-5 * (sum of |terms|) + 1e-6;
* the autograd chain (centre of mass, quaternion, per-type eps and rmin/2,
  site charges) against the same chain driven by the oracle's FP64 gradient,
  and that FP64 reference against central finite differences of FP64
  energies (h = 1e-4 A, 1e-4 on quaternion components, 1e-5 relative on
  parameters).
"""
import numpy as np
import pytest
import torch

from pygcmc_b200 import poses as PZ

pytestmark = pytest.mark.gpu

GRAD_REL = 1e-5


@pytest.fixture(scope="module")
def eng(protein_small):
    from pygcmc_b200.engine import Engine
    e = Engine(protein_small.copy())
    yield e
    e.close()


def well_conditioned(oracle_lib, s, xyz, q, t, cen, limit=1e8):
    _, _, _, El1 = oracle_lib.energy_batch(s, xyz.astype(np.float32), q.astype(np.float32), t, cen, mode=0,
                                           want_l1=True)
    return El1 < limit, El1


@pytest.mark.parametrize("ftype", [0, 3, 6])
def test_kernel_gradients_match_fp64_oracle(oracle_lib, eng, protein_small, ftype):
    from pygcmc_b200.grad import pose_energy
    s = protein_small
    tpl, q, t = PZ.template(s, ftype)
    com, quat = PZ.random_poses(s, 320, seed=10 + ftype)
    # random centres include near-coincident atom/site pairs whose FP32 terms
    # overflow (as the reference's FP32 calcEnergy does); keep the poses whose
    # sum of |pair terms| is representable with margin in FP32
    ok, _ = well_conditioned(oracle_lib, s, PZ.rigid_sites(tpl, com, quat), q.astype(np.float64), t,
                             com.astype(np.float32), limit=1e25)
    com, quat = com[ok][:256], quat[ok][:256]
    x32 = PZ.rigid_sites(tpl, com, quat).astype(np.float32)
    cen = com.astype(np.float32)
    dev = torch.device("cuda")
    X = torch.tensor(x32, device=dev, requires_grad=True)
    Q = torch.tensor(q, device=dev, requires_grad=True)
    F = torch.tensor(s.ff, device=dev, requires_grad=True)
    w = np.random.default_rng(ftype).normal(size=len(x32))
    E = pose_energy(eng, 0, X, Q, F, t, centres=torch.tensor(cen, device=dev))
    (E * torch.tensor(w, device=dev)).sum().backward()
    # energies equal the plain pose-energy path bit for bit (same kernel, same table)
    e_plain, _ = eng.energy_poses(x32, q, t, cen)
    assert np.array_equal(E.detach().cpu().numpy(), e_plain)
    ref = oracle_lib.grad_batch(s, x32.astype(np.float64), q.astype(np.float64), t, cen, gout=w)
    gx = X.grad.cpu().numpy().astype(np.float64)
    gx_ref = ref["gxyz"] * w[:, None, None]
    tol = GRAD_REL * np.abs(w)[:, None, None] * ref["gxyz_l1"][:, :, None] + 1e-6
    bad = np.argwhere(~(np.abs(gx - gx_ref) <= tol))
    for p, si, c in bad[:8]:
        print("bad", p, si, c, gx[p, si, c], gx_ref[p, si, c], tol[p, si, 0], ref["gxyz_l1"][p, si], w[p])
    assert len(bad) == 0, float((np.abs(gx - gx_ref) / tol).max())
    gq = Q.grad.cpu().numpy().astype(np.float64)
    gq_ref = (ref["gq"] * w[:, None]).sum(0)
    gq_l1 = (ref["gq_l1"] * np.abs(w)[:, None]).sum(0)
    assert np.all(np.abs(gq - gq_ref) <= GRAD_REL * gq_l1 + 1e-6)
    gf = F.grad.cpu().numpy().astype(np.float64)
    # ff is float32: the FP64 oracle table gradient is w.r.t. the same entries
    assert np.all(np.abs(gf - ref["gff"]) <= GRAD_REL * ref["gff_l1"] + 1e-6), \
        float((np.abs(gf - ref["gff"]) / (GRAD_REL * ref["gff_l1"] + 1e-6)).max())
    err = np.abs(gx - gx_ref) / np.maximum(np.abs(w)[:, None, None] * ref["gxyz_l1"][:, :, None], 1e-30)
    print(f"ftype {ftype}: max |dE/dx gpu - fp64| / l1 = {err.max():.2e}")


def _chain(system, ftype, com, quat, eps, rmin, charges, w, gxyz, gq, gff):
    """Back-propagate per-site/charge/table gradients through the rigid-pose and
    combining-rule chain in float64 on the CPU."""
    from pygcmc_b200.grad import lj_table, quat_to_matrix
    tpl, _, _ = PZ.template(system, ftype)
    c = torch.tensor(com, dtype=torch.float64, requires_grad=True)
    qt = torch.tensor(quat, dtype=torch.float64, requires_grad=True)
    e = torch.tensor(eps, dtype=torch.float64, requires_grad=True)
    r = torch.tensor(rmin, dtype=torch.float64, requires_grad=True)
    ch = torch.tensor(charges, dtype=torch.float64, requires_grad=True)
    sites = c[:, None, :] + torch.einsum("pij,sj->psi", quat_to_matrix(qt), torch.tensor(tpl))
    ffx = int(system.SimInfo[0]["ffXNum"])
    ff = lj_table(e, r, ffx)
    wt = torch.tensor(w, dtype=torch.float64)
    torch.autograd.backward([sites, ch, ff], [torch.tensor(gxyz) * wt[:, None, None],
                                              (torch.tensor(gq) * wt[:, None]).sum(0), torch.tensor(gff)])
    return c.grad.numpy(), qt.grad.numpy(), e.grad.numpy(), r.grad.numpy(), ch.grad.numpy()


def test_autograd_chain_matches_fp64_reference_and_finite_differences(oracle_lib, eng, protein_small):
    from pygcmc_b200.grad import RigidFragment, lj_table
    s = protein_small
    ftype = 1
    dev = torch.device("cuda")
    lt = s.meta["lj_types"]
    ffx = int(s.SimInfo[0]["ffXNum"])
    tpl, q0, t = PZ.template(s, ftype)
    com, quat = PZ.random_poses(s, 400, seed=21)
    # finite differences need energies whose rounding is small against the
    # change a 1e-5 relative parameter step makes: poses without deep clashes
    ok, El1 = well_conditioned(oracle_lib, s, PZ.rigid_sites(tpl, com, quat), q0.astype(np.float64), t,
                               com.astype(np.float32), limit=1e5)
    com, quat, El1 = com[ok][:64], quat[ok][:64], El1[ok][:64]
    assert len(com) == 64
    w = np.random.default_rng(4).normal(size=len(com))
    # GPU autograd
    frag = RigidFragment(eng, 0, ftype)
    C = torch.tensor(com, device=dev, requires_grad=True)
    Qt = torch.tensor(quat, device=dev, requires_grad=True)
    Ep = torch.tensor(lt["eps_kcal"], device=dev, requires_grad=True)
    Rm = torch.tensor(lt["rmin_half"], device=dev, requires_grad=True)
    Ch = torch.tensor(q0.astype(np.float64), device=dev, requires_grad=True)
    ff = lj_table(Ep, Rm, ffx)
    assert np.array_equal(ff.detach().float().cpu().numpy(), s.ff)
    E = frag.energy(C, Qt, ff, charges=Ch)
    (E * torch.tensor(w, device=dev)).sum().backward()
    g_gpu = [x.grad.cpu().numpy() for x in (C, Qt, Ep, Rm, Ch)]
    # FP64 reference: the oracle's analytic gradient at the kernels' float32 sites, chained in float64
    x32 = frag.sites(C.detach(), Qt.detach()).float().cpu().numpy()
    cen = com.astype(np.float32)
    ref = oracle_lib.grad_batch(s, x32.astype(np.float64), q0.astype(np.float64), t, cen, gout=w)
    g_ref = _chain(s, ftype, com, quat, lt["eps_kcal"], lt["rmin_half"], q0.astype(np.float64), w, ref["gxyz"],
                   ref["gq"], ref["gff"])
    # l1 scales of each gradient from the same chain driven by the |terms| sums
    sc = _chain(s, ftype, com, quat, lt["eps_kcal"], lt["rmin_half"], q0.astype(np.float64), np.abs(w),
                np.repeat(ref["gxyz_l1"][:, :, None], 3, axis=2), ref["gq_l1"], ref["gff_l1"])
    # quaternion: |d(R t)/dq_i| <= 4 |t| for a unit q, so bound by 4 sum_s |t_s| l1_s per pose
    tn = np.linalg.norm(tpl, axis=1)
    sc = list(sc)
    sc[1] = np.repeat((4 * np.abs(w) * (ref["gxyz_l1"] * tn[None, :]).sum(1))[:, None], 4, axis=1)
    names = ["com", "quat", "eps", "rmin", "charge"]
    for name, a, b, m in zip(names, g_gpu, g_ref, sc):
        bound = 4 * GRAD_REL * np.abs(m) + 1e-6
        assert np.all(np.abs(a - b) <= bound), (name, float((np.abs(a - b) / bound).max()))
    # FP64 reference gradient vs central differences of FP64 energies of float64 sites
    x64 = PZ.rigid_sites(tpl, com, quat)
    ref64 = oracle_lib.grad_batch(s, x64, q0.astype(np.float64), t, cen, gout=w)
    g64 = _chain(s, ftype, com, quat, lt["eps_kcal"], lt["rmin_half"], q0.astype(np.float64), w, ref64["gxyz"],
                 ref64["gq"], ref64["gff"])

    def loss(com_, quat_, eps_, rmin_, ch_):
        ff64 = lj_table(torch.tensor(eps_), torch.tensor(rmin_), ffx).numpy()
        e, ng = oracle_lib.energy_batch64(s, PZ.rigid_sites(tpl, com_, quat_), ch_, t, com_.astype(np.float32),
                                          ff=ff64)
        return e, ng

    args = [com, quat, lt["eps_kcal"].astype(np.float64), lt["rmin_half"].astype(np.float64), q0.astype(np.float64)]
    _, ng0 = loss(*args)
    checked = 0
    for which, h_abs, h_rel in ((0, 1e-4, None), (1, 1e-4, None), (2, None, 1e-5), (3, None, 1e-5), (4, None, 1e-5)):
        base = args[which]
        flat = base.reshape(-1)
        idx = range(len(flat)) if which >= 2 else np.random.default_rng(which).choice(len(flat), 24, replace=False)
        for j in idx:
            h = h_abs if h_abs is not None else h_rel * abs(flat[j])
            if h == 0:
                continue
            ap, am = [a.copy() for a in args], [a.copy() for a in args]
            ap[which].reshape(-1)[j] += h
            am[which].reshape(-1)[j] -= h
            ep, ngp = loss(*ap)
            em, ngm = loss(*am)
            keep = (ngp == ng0) & (ngm == ng0)  # inclusion unchanged by the step
            if which <= 1:  # com / quat entries belong to one pose
                p = j // base.shape[1]
                if not keep[p]:
                    continue
                fd = w[p] * (ep[p] - em[p]) / (2 * h)
                rounding = 64 * 2.2e-16 * abs(w[p]) * El1[p] / (2 * h)
            else:
                if not keep.all():
                    continue
                fd = w @ (ep - em) / (2 * h)
                rounding = 64 * 2.2e-16 * (np.abs(w) @ El1) / (2 * h)
            an = g64[which].reshape(-1)[j]
            scale = np.abs(sc[which].reshape(-1)[j])
            # central-difference truncation (relative to the l1 scale) plus the energies' rounding
            assert abs(fd - an) <= 1e-5 * scale + rounding + 1e-9, (names[which], j, fd, an, scale, rounding)
            checked += 1
    assert checked > 80
