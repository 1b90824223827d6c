"""Differentiable pose energies (PyTorch autograd over gcmc_energy_grad).

:class:`PoseEnergy` maps explicit poses -- site coordinates, site charges and
the LJ pair table in the reference's layout (sigma [nm], eps [kJ/mol] per
(site type, atom type); gcmc/cpp/gcmc_energy.h:160-161) -- to the FP64 pose
energies of the engine's kernels, and its backward calls the hand-written
gradient kernel.  :class:`RigidFragment` builds the sites of a fragment type
from a centre of mass and a quaternion, and :func:`lj_table` the pair table
from per-type CHARMM parameters with the reference's combining rule
(gcmc/python/simulation.py:56-75), so that autograd reaches
d E / d(centre of mass, quaternion, eps, rmin/2, site charges).

The environment (fixed atoms and occupied fragment slots of the replica) is
the engine's current state and carries no gradient.  Group inclusion is by
pose centre (the centre of mass), a hard cutoff: E is smooth in the site
coordinates and parameters, piecewise constant in which groups count.
"""
import ctypes

import numpy as np
import torch

from . import values as V
from ._native import check, lib


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream():
    """torch's current stream as a cudaStream_t.  torch reports the legacy
    default stream as 0, which the C ABI reads as "the context's stream"; pass
    cudaStreamLegacy (0x1) instead so the kernels stay ordered with torch's work."""
    h = torch.cuda.current_stream().cuda_stream
    return ctypes.c_void_p(h if h else 1)


class PoseEnergy(torch.autograd.Function):
    """E[p] (float64) of poses ``xyz`` [P, ns, 3] float32 with charges ``q`` [ns]
    float32 and pair table ``ff`` [ffX*ffY*2] float32 (all CUDA); ``centres``
    [P, 3] float32 selects the included groups (no gradient)."""

    @staticmethod
    def forward(ctx, xyz, q, ff, centres, engine, rep, site_type, site_type_dev, self_res):
        xyz = xyz.contiguous()
        q = q.contiguous()
        ff = ff.contiguous()
        centres = centres.contiguous()
        P, ns = xyz.shape[0], xyz.shape[1]
        E = torch.empty(P, dtype=torch.float64, device=xyz.device)
        check(lib().gcmc_energy_grad(engine.handle, rep, _p(xyz), _p(q), _p(site_type_dev),
                                     site_type.ctypes.data_as(ctypes.c_void_p), ns, _p(centres), _p(self_res), P,
                                     _p(ff), None, _p(E), None, None, None, _stream()), "gcmc_energy_grad")
        ctx.save_for_backward(xyz, q, ff, centres)
        ctx.engine, ctx.rep, ctx.site_type, ctx.site_type_dev, ctx.self_res = (engine, rep, site_type,
                                                                                site_type_dev, self_res)
        return E

    @staticmethod
    def backward(ctx, gE):
        xyz, q, ff, centres = ctx.saved_tensors
        P, ns = xyz.shape[0], xyz.shape[1]
        gE = gE.detach().to(torch.float64).contiguous()
        need_x, need_q, need_ff = ctx.needs_input_grad[0], ctx.needs_input_grad[1], ctx.needs_input_grad[2]
        gxyz = torch.empty((P, ns, 3), dtype=torch.float64, device=xyz.device) if need_x else None
        gq = torch.empty((P, ns), dtype=torch.float64, device=xyz.device) if need_q else None
        gff = torch.zeros(ff.shape[0], dtype=torch.float64, device=xyz.device) if need_ff else None
        if need_x or need_q or need_ff:
            check(lib().gcmc_energy_grad(ctx.engine.handle, ctx.rep, _p(xyz), _p(q), _p(ctx.site_type_dev),
                                         ctx.site_type.ctypes.data_as(ctypes.c_void_p), ns, _p(centres),
                                         _p(ctx.self_res), P, _p(ff), _p(gE), None, _p(gxyz), _p(gq), _p(gff),
                                         _stream()), "gcmc_energy_grad")
        gx = (gxyz * gE[:, None, None]).to(xyz.dtype) if need_x else None
        gqs = (gq * gE[:, None]).sum(0).to(q.dtype) if need_q else None
        gf = gff.to(ff.dtype) if need_ff else None
        return gx, gqs, gf, None, None, None, None, None, None


def pose_energy(engine, rep, xyz, q, ff, site_type, centres=None, self_res=None):
    """Differentiable E[p] for sites ``xyz`` [P, ns, 3] (any float dtype; the
    kernels see float32), charges ``q`` [ns], table ``ff``; ``site_type`` a
    numpy int32 array [ns].  ``centres`` defaults to the site centroids."""
    dev = xyz.device
    st = np.ascontiguousarray(site_type, dtype=np.int32)
    st_dev = torch.from_numpy(st).to(dev)
    if centres is None:
        centres = xyz.detach().mean(dim=1)
    sr = None if self_res is None else torch.as_tensor(self_res, dtype=torch.int32, device=dev).contiguous()
    return PoseEnergy.apply(xyz.to(torch.float32), q.to(torch.float32), ff.to(torch.float32),
                            centres.detach().to(torch.float32), engine, int(rep), st, st_dev, sr)


def quat_to_matrix(q):
    """Rotation matrices [..., 3, 3] of quaternions q [..., 4] = (w, x, y, z),
    normalised first (so gradients are tangent to the unit sphere)."""
    q = q / q.norm(dim=-1, keepdim=True)
    w, x, y, z = q.unbind(-1)
    return torch.stack([
        torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        torch.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        torch.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], -2)


def lj_table(eps_kcal, rmin_half, n_rows: int):
    """Pair table (sigma [nm], eps [kJ/mol]) [n_rows * n * 2] from per-type
    CHARMM eps [kcal/mol] and rmin/2 [A] (n types, the first n_rows being the
    fragment site types): sigma = 2 rmin/2 / 2^(1/6) / 10, eps_kJ = 4.184 eps,
    Lorentz-Berthelot combining (gcmc/python/simulation.py:64-72)."""
    sigma = 2.0 * rmin_half / 2.0 ** (1.0 / 6.0) / 10.0
    e = V.KCAL_TO_KJ * eps_kcal
    s2 = (sigma[:n_rows, None] + sigma[None, :]) / 2
    e2 = torch.sqrt(e[:n_rows, None] * e[None, :])
    return torch.stack([s2, e2], -1).reshape(-1)


class RigidFragment:
    """Poses of fragment type ``ftype`` of replica ``rep`` of an Engine:
    x_s = com + R(quat) (t_s - mean t)."""

    def __init__(self, engine, rep: int, ftype: int, device="cuda", dtype=torch.float64):
        from . import poses as PZ
        tpl, q, t = PZ.template(engine.systems[rep], ftype)
        self.engine, self.rep, self.ftype = engine, rep, ftype
        self.template = torch.as_tensor(tpl, dtype=dtype, device=device)
        self.charges = torch.as_tensor(q, dtype=dtype, device=device)
        self.site_type = t

    def sites(self, com, quat):
        R = quat_to_matrix(quat)
        return com[:, None, :] + torch.einsum("pij,sj->psi", R, self.template.to(com.dtype))

    def energy(self, com, quat, ff, charges=None):
        q = self.charges if charges is None else charges
        return pose_energy(self.engine, self.rep, self.sites(com, quat), q, ff, self.site_type,
                           centres=com.detach())
