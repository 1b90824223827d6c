"""Parameter sensitivities of the fragment occupancy from a GCMC run.

In the grand-canonical ensemble, for a parameter theta of the potential U,
    d<N_t>/d theta = -beta ( <N_t dU/dtheta> - <N_t> <dU/dtheta> ),
with N_t the number of fragments of type t.  dU/dtheta of a configuration
comes from the backward kernel (gcmc_energy_grad) applied to every occupied
fragment as an explicit pose against the rest of the state:

* site charges: the sum over fragments of dE_f/dq_s is dU/dq_s exactly (each
  pose differentiates only its own sites' charges);
* per-type eps and rmin/2 (through the Lorentz-Berthelot pair table): the sum
  over fragments counts fragment-fragment pairs from both ends, so
  dU/dtheta = (S_all + S_fixed) / 2 with S_fixed the same sum against the
  fixed atoms alone (a context of the snapshot with no fragments).

Parameters that only change fixed-fixed interactions give a constant dU/dtheta
and drop out of the covariance.
"""
import numpy as np
import torch

from .values import Info_dtype  # noqa: F401  (structured arrays of the state)

BETA = 1.0 / (0.0083115 * 300.0)  # mol/kJ at the reference's T and k_B


def _occupied(system):
    """Per type: (site xyz [n, ns, 3], centres [n, 3], residue ids [n])."""
    out = []
    for f in system.fragmentInfo:
        ns, n, s0 = int(f["num_atoms"]), int(f["totalNum"]), int(f["startRes"])
        res = system.residueInfo[s0:s0 + n]
        idx = res["atomStart"][:, None] + np.arange(ns)[None, :]
        out.append((system.atomInfo["position"][idx].astype(np.float32), res["position"].astype(np.float32),
                    np.arange(s0, s0 + n, dtype=np.int32)))
    return out


def configuration_gradient(engine, state, eps_kcal, rmin_half, rep: int = 0):
    """dU/dtheta of the engine's current configuration ``state`` (its download)
    for theta = (per-type eps [kcal/mol], per-type rmin/2 [A], site charges of
    each fragment type).  Returns (g_eps, g_rmin, [g_q per type])."""
    from ._native import default_options
    from .engine import Engine
    from .grad import lj_table, pose_energy
    dev = torch.device("cuda")
    ffx = int(state.SimInfo[0]["ffXNum"])
    empty = state.copy()
    empty.fragmentInfo["totalNum"] = 0
    sums = {}
    with Engine(empty, default_options()) as fixed_only:
        for which, eng in (("all", engine), ("fixed", fixed_only)):
            e = torch.tensor(eps_kcal, dtype=torch.float64, device=dev, requires_grad=True)
            r = torch.tensor(rmin_half, dtype=torch.float64, device=dev, requires_grad=True)
            ff = lj_table(e, r, ffx)
            total = torch.zeros((), dtype=torch.float64, device=dev)
            qs = []
            for t, (xyz, cen, self_res) in enumerate(_occupied(state)):
                f = state.fragmentInfo[t]
                ns = int(f["num_atoms"])
                q = torch.tensor(f["atoms"]["charge"][:ns].astype(np.float64), device=dev, requires_grad=True)
                qs.append(q)
                if len(xyz) == 0:
                    continue
                E = pose_energy(eng, rep if which == "all" else 0, torch.tensor(xyz, device=dev), q, ff,
                                f["atoms"]["type"][:ns].astype(np.int32), centres=torch.tensor(cen, device=dev),
                                self_res=self_res)
                total = total + E.sum()
            if total.requires_grad:
                total.backward()
            sums[which] = (e.grad.cpu().numpy() if e.grad is not None else np.zeros(len(eps_kcal)),
                           r.grad.cpu().numpy() if r.grad is not None else np.zeros(len(rmin_half)),
                           [q.grad.cpu().numpy() if q.grad is not None else np.zeros(len(q)) for q in qs])
    ge = 0.5 * (sums["all"][0] + sums["fixed"][0])
    gr = 0.5 * (sums["all"][1] + sums["fixed"][1])
    return ge, gr, sums["all"][2]


def occupancy_sensitivity(system, options, nsamples: int, stride: int, eps_kcal, rmin_half, burn: int = 0):
    """Run ``system`` and estimate d<N_t>/d(eps, rmin/2, site charges) from
    ``nsamples`` snapshots taken every ``stride`` MC steps after ``burn`` steps.
    Returns a dict with the mean counts, the sensitivities (arrays indexed
    [type, parameter]) and their per-sample inputs."""
    from .engine import Engine
    N, G_e, G_r, G_q = [], [], [], []
    with Engine(system.copy(), options) as eng:
        if burn:
            eng.run(burn)
        for _ in range(nsamples):
            eng.run(stride)
            eng.sync()
            state = eng.download()
            ge, gr, gq = configuration_gradient(eng, state, eps_kcal, rmin_half)
            N.append(state.fragmentInfo["totalNum"].astype(np.float64))
            G_e.append(ge)
            G_r.append(gr)
            G_q.append(np.concatenate(gq))
    N, G_e, G_r, G_q = map(np.asarray, (N, G_e, G_r, G_q))

    def cov(a, b):
        return (a[:, :, None] * b[:, None, :]).mean(0) - a.mean(0)[:, None] * b.mean(0)[None, :]

    return {"mean_N": N.mean(0), "dN_deps": -BETA * cov(N, G_e), "dN_drmin": -BETA * cov(N, G_r),
            "dN_dq": -BETA * cov(N, G_q), "samples": {"N": N, "dU_deps": G_e, "dU_drmin": G_r, "dU_dq": G_q}}
